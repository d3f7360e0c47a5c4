"""TEST INFRASTRUCTURE ONLY: FP64 numpy restatement of the warm-start CNN's
convolutions (3x3, stride 1, zero padding, NHWC, weights [co][9][ci] with
tap = 3*dy + dx), their data and weight gradients, and BF16 rounding.  Used
by tests/ to check ctlab_cnn_* kernels; never by the product path.

The CNN has no counterpart in the reference (it is the learned warm start
of OS-SART); this restates the standard convolution algebra."""
import numpy as np


def bf16(a):
    """Round to bfloat16 (nearest even), returned as float32 values."""
    x = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((x + 0x7FFF + ((x >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(np.shape(a))


def bf16_bits(a):
    """bfloat16 bit patterns (uint16) of bf16(a)."""
    return (bf16(a).view(np.uint32) >> 16).astype(np.uint16)


def conv3x3(x, w, b=None):
    """x [B,H,W,CI], w [CO,9,CI] -> [B,H,W,CO] in FP64."""
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    B, H, W, CI = x.shape
    xp = np.zeros((B, H + 2, W + 2, CI))
    xp[:, 1:-1, 1:-1] = x
    out = np.zeros((B, H, W, w.shape[0]))
    for t in range(9):
        dy, dx = divmod(t, 3)
        out += np.einsum("bhwc,oc->bhwo", xp[:, dy:dy + H, dx:dx + W], w[:, t, :])
    if b is not None:
        out += np.asarray(b, np.float64)
    return out


def flip_transpose(w):
    """Weights of the data-gradient convolution: wt[ci][8 - t][co] = w[co][t][ci]."""
    return np.ascontiguousarray(np.transpose(np.asarray(w)[:, ::-1, :], (2, 1, 0)))


def conv_wgrad(dpre, act):
    """dW[co][t][ci] = sum_p dpre[p][co] act[p + tap(t)][ci] (FP64)."""
    d = np.asarray(dpre, np.float64)
    a = np.asarray(act, np.float64)
    B, H, W, CI = a.shape
    ap = np.zeros((B, H + 2, W + 2, CI))
    ap[:, 1:-1, 1:-1] = a
    dw = np.zeros((d.shape[3], 9, CI))
    for t in range(9):
        dy, dx = divmod(t, 3)
        dw[:, t, :] = np.einsum("bhwo,bhwc->oc", d, ap[:, dy:dy + H, dx:dx + W])
    return dw
