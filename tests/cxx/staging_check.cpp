// Prints the z-prefix projector staging the library's host planner picks for
// each scan read from stdin (one ctlab_geometry per record: 14 scalars, then
// xds, yds, zds, hangs, hzPos), for the staging invariants test.  Host only.
#include <cstdio>
#include <vector>

#include "../../ctlab_b200/csrc/internal.h"

using namespace ctlab;

int main()
{
    for (int idx = 0;; ++idx) {
        ctlab_geometry g;
        int DNU, DNV, PN;
        if (std::scanf("%f %f %f %d %d %d %d %d %d %f %f %f %f %f", &g.x0, &g.y0, &g.z0, &DNU, &DNV, &PN, &g.XN, &g.YN,
                       &g.ZN, &g.dx, &g.dz, &g.imgXCenter, &g.imgYCenter, &g.imgZCenter) != 14)
            return 0;
        g.DNU = DNU;
        g.DNV = DNV;
        g.PN = PN;
        std::vector<float> xds(DNU), yds(DNU), zds(DNV), h(PN), hz(PN);
        for (std::vector<float> *a : {&xds, &yds, &zds, &h, &hz})
            for (float &v : *a)
                if (std::scanf("%f", &v) != 1) return 2;
        g.xds = xds.data();
        g.yds = yds.data();
        g.zds = zds.data();
        g.hangs = h.data();
        g.hzPos = hz.data();
        HostGeometry hg;
        if (build_geometry(g, hg) != CTLAB_OK) return 3;
        for (int wcap : {15, 7})
        for (int gcap : {16, 1}) {
            const ProjTStaging st = proj_t_staging(hg, gcap, 0, 0, wcap);
            std::vector<int> all(PN);
            for (int i = 0; i < PN; ++i) all[i] = i;
            const ProjGroups pg = proj_t_make_groups(hg, all, st);
            int nr = 0, rb = 0;
            proj_t_split(st, pg.G, nr, rb);
            // every list position exactly once in the table (-1 pads a group)
            std::vector<int> seen(PN, 0);
            int bad = 0;
            for (int q : pg.table) {
                if (q < -1 || q >= PN) ++bad;
                else if (q >= 0) ++seen[q];
            }
            for (int c : seen) bad += c != 1;
            std::printf("%d %d ok=%d G=%d NR=%d RB=%d ZS=%d CB=%d KB=%d KR=%d nstage=%d smem=%zu groupsG=%d ngroups=%d "
                        "table=%zu lnr=%d lrb=%d DNV=%d PN=%d badpos=%d W=%d\n",
                        idx, gcap, (int)st.ok, st.G, st.NR, st.RB, st.ZS, st.CB, st.KB, st.KR, st.nstage, st.smem, pg.G,
                        pg.ngroups, pg.table.size(), nr, rb, DNV, PN, bad, st.W);
        }
    }
}
