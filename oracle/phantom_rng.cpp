// TEST INFRASTRUCTURE ONLY.  The seeded random-ellipsoid sampler of the
// synthetic workloads, restated for the oracle so that the CPU baseline and
// the tests can draw phantoms without loading the CUDA library.  Same engine
// (std::mt19937_64 seeded with `seed`), same distributions and the same order
// of draws as ctlab_random_ellipsoids: count ~ U{n_min..n_max}; per ellipsoid
// centre x, y, z ~ U(-0.8, 0.8) x half extent, semi-axes ~ U(0.05, 0.4) x
// half extent, three Euler angles ~ U(0, pi), value ~ U(0, v_max).  Records
// are 10 doubles: value, centre (3), semi-axes (3), angles (3).
#include <algorithm>
#include <cmath>
#include <random>

extern "C" int orc_random_ellipsoids(unsigned long long seed, int n_min, int n_max, float half_x, float half_y,
                                     float half_z, float v_max, double *out, int cap)
{
    if (!out || n_min < 1 || n_max < n_min || cap < 1) return -1;
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<int> count(n_min, n_max);
    std::uniform_real_distribution<double> unit(0.0, 1.0);
    const int n = std::min(count(rng), cap);
    const double h[3] = {half_x, half_y, half_z};
    for (int e = 0; e < n; ++e) {
        double *E = out + 10 * e;
        for (int a = 0; a < 3; ++a) E[1 + a] = (2.0 * unit(rng) - 1.0) * 0.8 * h[a];
        for (int a = 0; a < 3; ++a) E[4 + a] = (0.05 + 0.35 * unit(rng)) * h[a];
        for (int a = 0; a < 3; ++a) E[7 + a] = unit(rng) * M_PI;
        E[0] = unit(rng) * (double)v_max;
    }
    return n;
}
