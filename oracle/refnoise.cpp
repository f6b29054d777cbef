/*
 * refnoise.cpp -- the reference's Gaussian stream, for parity fixtures.
 * TEST INFRASTRUCTURE ONLY.
 *
 * The reference draws its noise from one std::mt19937_64 seeded with
 * seed + llround(restart/dt) (init.cpp:402-413, init_random) through one
 * std::normal_distribution<double>(0, 1) (init.cpp:105-110): per step nm3nc11
 * draws for the slip noise (slip_vel.cpp:11-17), then nm3nc6 for the RFD
 * direction (drift.cpp:9-15).  Built with the same C++ standard library as the
 * reference module, this returns the first n draws of that stream.
 */
#include <random>

extern "C" void ref_normals(unsigned long seed, long n, double *out)
{
    std::mt19937_64 rng;
    rng.seed(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    for (long i = 0; i < n; i++) out[i] = nd(rng);
}
