// lj_host_init.cpp -- host-side initial condition (engine::InitialCondition).
//
// The initial state stays on the host because the seed contract is libstdc++'s
// std::mt19937 + std::normal_distribution (engine/initial_condition.cpp:76-86);
// it is built once and uploaded.
//   * FCC lattice sites in x-major, y, z, sub-site order, scaled to the density
//     (tools/cubic_lattice.cpp:38-86)
//   * Maxwell-Boltzmann velocities, one normal draw per component in the order
//     x0, y0, z0, x1, ... (initial_condition.cpp:76-86)
//   * zero momentum, zero angular momentum about the centre of mass, rescale
//     to T (initial_condition.cpp:96-101, transformations.cpp:35-116).  The
//     reference solves the 4x4 inertia system with Eigen's
//     fullPivHouseholderQr; its 4th row and column decouple, so a 3x3 solve
//     (Gaussian elimination with partial pivoting) gives the same solution up
//     to rounding.

#include <cmath>
#include <cstdlib>
#include <random>
#include <utility>
#include <vector>

#include "../../include/lj_gpu.h"


namespace {

void solve3(double A[3][3], double b[3], double w[3]) {
    int p[3] = {0, 1, 2};
    for (int c = 0; c < 3; ++c) {
        int best = c;
        for (int r = c + 1; r < 3; ++r)
            if (std::fabs(A[p[r]][c]) > std::fabs(A[p[best]][c])) best = r;
        std::swap(p[c], p[best]);
        for (int r = c + 1; r < 3; ++r) {
            double m = A[p[r]][c] / A[p[c]][c];
            for (int k = c; k < 3; ++k) A[p[r]][k] -= m * A[p[c]][k];
            b[p[r]] -= m * b[p[c]];
        }
    }
    for (int c = 2; c >= 0; --c) {
        double acc = b[p[c]];
        for (int k = c + 1; k < 3; ++k) acc -= A[p[c]][k] * w[k];
        w[c] = acc / A[p[c]][c];
    }
}

constexpr double kFcc[4][3] = {{0.0, 0.0, 0.0}, {0.5, 0.5, 0.0}, {0.5, 0.0, 0.5}, {0.0, 0.5, 0.5}};

}  // namespace

extern "C" int lj_initial_condition(int N, double temperature, double density, unsigned seed,
                                    double* x, double* v, double* side) {
    if (N < 1 || !(density > 0) || !(temperature > 0) || !x || !v || !side) return LJ_ERR_ARG;
    // tools/cubic_lattice.cpp:43-58
    int nonempty = (int)std::ceil((double)N / 4.0);
    int cps = (int)std::ceil(std::cbrt((double)nonempty));
    double proto = (double)N / (double)(cps * cps * cps);
    double scale = std::cbrt(proto / density);
    *side = (double)cps * scale;
    // tools/cubic_lattice.cpp:61-86
    for (int index = 0; index < N; ++index) {
        auto xyz_s = std::div(index, 4);
        auto xy_z = std::div(xyz_s.quot, cps);
        auto x_y = std::div(xy_z.quot, cps);
        int cell[3] = {x_y.quot, x_y.rem, xy_z.rem};
        for (int k = 0; k < 3; ++k) x[4 * (size_t)index + k] = ((double)cell[k] + kFcc[xyz_s.rem][k]) * scale;
        x[4 * (size_t)index + 3] = 0.0;
    }
    std::mt19937 gen{seed};
    std::normal_distribution<> mb{0, std::sqrt(temperature)};
    for (int i = 0; i < N; ++i) {
        for (int k = 0; k < 3; ++k) v[4 * (size_t)i + k] = mb(gen);
        v[4 * (size_t)i + 3] = 0.0;
    }
    double com[3] = {0, 0, 0}, p[3] = {0, 0, 0};
    for (int i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) {
            com[k] += x[4 * (size_t)i + k];
            p[k] += v[4 * (size_t)i + k];
        }
    for (int k = 0; k < 3; ++k) {
        com[k] /= (double)N;
        double dv = (0.0 - p[k]) / (double)N;
        for (int i = 0; i < N; ++i) v[4 * (size_t)i + k] += dv;
    }
    double I[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, L[3] = {0, 0, 0};
    for (int i = 0; i < N; ++i) {
        double r[3], u[3];
        for (int k = 0; k < 3; ++k) {
            r[k] = x[4 * (size_t)i + k] - com[k];
            u[k] = v[4 * (size_t)i + k];
        }
        double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) I[a][b] += (a == b ? r2 : 0.0) - r[a] * r[b];
        L[0] += r[1] * u[2] - r[2] * u[1];
        L[1] += r[2] * u[0] - r[0] * u[2];
        L[2] += r[0] * u[1] - r[1] * u[0];
    }
    if (N > 1) {
        double rhs[3] = {-L[0], -L[1], -L[2]}, w[3] = {0, 0, 0};
        solve3(I, rhs, w);
        for (int i = 0; i < N; ++i) {
            double r[3];
            for (int k = 0; k < 3; ++k) r[k] = x[4 * (size_t)i + k] - com[k];
            v[4 * (size_t)i + 0] += w[1] * r[2] - w[2] * r[1];
            v[4 * (size_t)i + 1] += w[2] * r[0] - w[0] * r[2];
            v[4 * (size_t)i + 2] += w[0] * r[1] - w[1] * r[0];
        }
    }
    // set_temperature (transformations.cpp:94-116)
    double acc = 0;
    for (int i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) acc += v[4 * (size_t)i + k] * v[4 * (size_t)i + k];
    double T = (2. / 3.) * ((1. / 2.) * acc) / (double)N;
    if (!(T > 0)) return LJ_ERR_ARG;
    double f = std::sqrt(temperature / T);
    for (int i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) v[4 * (size_t)i + k] *= f;
    return LJ_OK;
}
