// Test program: calls the reference-signature C++ entry points of
// libctlab_b200 (OS_SART or CG over thrust::host_vector) on a scan read from
// a binary file and writes the reconstruction to a raw float32 file.
//   recon_caller <in.bin> <out.raw> <os|cg> [cg_method]
// in.bin: int32 DNU DNV PN XN YN ZN osNum iterNum, float32 sid sdd cx cy cz
// dx dz col_size row_size col_offset row_offset, then float32 hangs[PN],
// hzPos[PN], init[XN*YN*ZN], prj[PN*DNU*DNV] and uint8 mask[XN*YN].
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "ctlab_b200_recon.hpp"

template <class T>
static bool rd(FILE *f, T *p, size_t n) { return std::fread(p, sizeof(T), n, f) == n; }

int main(int argc, char **argv)
{
    if (argc < 4) return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int iv[8];
    float fv[11];
    if (!rd(f, iv, 8) || !rd(f, fv, 11)) return 2;
    const int DNU = iv[0], DNV = iv[1], PN = iv[2], XN = iv[3], YN = iv[4], ZN = iv[5], os = iv[6], it = iv[7];
    thrust::host_vector<float> hangs(PN), hzPos(PN), init((size_t)XN * YN * ZN), prj((size_t)PN * DNU * DNV), recon;
    thrust::host_vector<byte> mask((size_t)XN * YN);
    if (!rd(f, hangs.data(), hangs.size()) || !rd(f, hzPos.data(), hzPos.size()) || !rd(f, init.data(), init.size()) ||
        !rd(f, prj.data(), prj.size()) || !rd(f, mask.data(), mask.size()))
        return 2;
    std::fclose(f);
    const std::string out = argv[2];
    if (std::strcmp(argv[3], "os") == 0)
        OS_SART(recon, init, prj, hangs, hzPos, mask, out, os, it, false, fv[0], fv[1], DNU, DNV, PN, fv[2], fv[3],
                fv[4], XN, YN, ZN, fv[5], fv[6], fv[7], fv[8], fv[9], fv[10], PROJ_BRANCHLESS, BACK_BRANCHLESS);
    else
        CG(recon, init, prj, hangs, hzPos, mask, out, os, it, false, fv[0], fv[1], DNU, DNV, PN, fv[2], fv[3], fv[4],
           XN, YN, ZN, fv[5], fv[6], fv[7], fv[8], fv[9], fv[10], PROJ_BRANCHLESS, BACK_BRANCHLESS,
           (CGMethod)(argc > 4 ? std::atoi(argv[4]) : 0));
    if (ctlab_last_status() != CTLAB_OK) {
        std::fprintf(stderr, "%s\n", ctlab_last_error());
        return 1;
    }
    return recon.size() == init.size() ? 0 : 1;
}
