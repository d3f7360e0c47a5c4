"""The z-prefix projector's host planner (proj_t_staging, proj_t_make_groups,
proj_t_split in libctlab_b200.so) on the benchmark scans and on edge cases:
every staging respects the kernel's limits (rows per warp a multiple of 4 up to
32, <= 15 consumer warps, every detector row covered, shared memory within the
per-CTA limit, 16-byte TMA rows of (P, f) pairs) and every view lands in exactly one group.
Host only: the driver is compiled against the library, no GPU needed."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from ctlab_b200 import _lib
from ctlab_b200 import geometry as G

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cxx", "staging_check.cpp")


def scans():
    out = [G.config1(), G.config2(), G.config3()] + G.config4()
    out += [G.small(), G.small(DNV=1, row_size=0.5), G.small(DNU=9, DNV=5, col_size=4.0, row_size=3.0),
            G.small(PN=40, ZN=600, dz=0.05, zpos=np.linspace(-14.0, 14.0, 40)),
            G.small(XN=9, YN=8, ZN=300, DNU=20, DNV=40, dz=0.05, row_size=0.1),
            G.small(PN=7, DNV=200, row_size=0.05),
            G.helical(XN=64, YN=64, ZN=128, views_per_turn=96)]
    return out


def dump(gs):
    lines = []
    for g in gs:
        a = [g.x0, g.y0, g.z0, g.DNU, g.DNV, g.PN, g.XN, g.YN, g.ZN, g.dx, g.dz, g.imgXCenter, g.imgYCenter,
             g.imgZCenter]
        lines.append(" ".join(str(x) for x in a))
        for arr in (g.xds, g.yds, g.zds, g.hangs, g.hzPos):
            lines.append(" ".join("%.9g" % x for x in arr))
    return "\n".join(lines) + "\n"


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if not shutil.which("nvcc"):
        pytest.skip("nvcc not found")
    out = str(tmp_path_factory.mktemp("planner") / "staging_check")
    libdir = os.path.dirname(_lib.LIB_PATH)
    r = subprocess.run(["nvcc", "-std=c++17", "-x", "cu", "-gencode", "arch=compute_100a,code=sm_100a", SRC,
                        "-L" + libdir, "-lctlab_b200", "-Xlinker", "-rpath=" + libdir, "-o", out],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return out


def test_stagings_respect_the_kernel_limits(driver):
    gs = scans()
    r = subprocess.run([driver], input=dump(gs), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    rows = [dict(re.findall(r"(\w+)=(\d+)", l)) | {"idx": l.split()[0], "gcap": l.split()[1]}
            for l in r.stdout.splitlines()]
    assert len(rows) == 4 * len(gs)  # 16- and 8-warp CTAs, 16 views and 1 view per CTA
    for d in rows:
        v = {k: int(x) for k, x in d.items()}
        assert v["ok"] == 1
        W = v["W"]
        assert W in (15, 7), d
        assert v["NR"] % 4 == 0 and 4 <= v["NR"] <= 32, d
        assert v["G"] * v["RB"] <= W and v["G"] >= 1, d
        assert v["NR"] * v["RB"] * v["ZS"] >= v["DNV"], d          # every detector row covered
        assert v["lnr"] * v["lrb"] == v["NR"] * v["RB"], d         # the launch split keeps the rows
        assert v["lnr"] % 4 == 0 and v["groupsG"] * v["lrb"] <= W, d
        # one CTA within the SM's limit; two 8-warp CTAs within half of it each
        assert v["smem"] + 14 * 1024 <= (227 * 1024 if W == 15 else 227 * 1024 // 2 - 1024) or v["CB"] == 0, d
        if v["CB"]:
            # 16-byte rows of 8-byte (P, f) pairs, 128-byte aligned boxes
            assert v["CB"] % 2 == 0 and (v["KB"] * v["CB"]) % 16 == 0 and v["KR"] % v["KB"] == 0, d
        assert v["groupsG"] <= v["G"] and v["table"] == v["ngroups"] * v["groupsG"], d
        if v["gcap"] == 1:
            assert v["G"] == 1, d


def test_every_view_is_grouped_once(driver):
    gs = scans()
    r = subprocess.run([driver], input=dump(gs), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    for l in r.stdout.splitlines():
        v = {k: int(x) for k, x in re.findall(r"(\w+)=(\d+)", l)}
        assert v["badpos"] == 0, l
