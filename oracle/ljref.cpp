/*
 * ljref.cpp -- CPU oracle for the Lennard-Jones NVE hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a single-threaded CPU restatement of
 * bniehoff/lennard-jonesium's hot path.  Only the tests, the smoke check and the
 * CPU-baseline leg of the benchmark load it, and only as the checker or as the
 * timed CPU baseline.  The GPU library never links or calls it.
 *
 * The reference itself cannot be compiled here (it needs Eigen 3.4, Boost and
 * Catch2, none of which exist in this image), so this is a restatement that
 * follows the arithmetic of the cited reference lines.  Where the reference
 * leaves an order open (Eigen reductions under -ffast-math), the order used
 * here is fixed and documented, and the GPU FP64 path uses the same order for
 * everything that must be bit-exact (cell index, separation, r^2 and the
 * cutoff test).
 *
 * Fixed orders (shared with the GPU FP64 path):
 *   separation  s_k = (x_i,k - x_j,k) - image_k * L_k
 *       (engine/particle_pair_filter.cpp:180-183, left to right)
 *   r^2         fma(s_z, s_z, fma(s_y, s_y, s_x * s_x))
 *   in cutoff   r^2 < rc*rc              (particle_pair_filter.cpp:185)
 *   cell index  clamp(floor(x_k * (n_k / L_k)), 0, n_k - 1)
 *       (particle_pair_filter.cpp:144-147; the clamp only changes cases that
 *        are out of bounds, i.e. undefined behaviour, in the reference)
 *
 * The oracle is pinned against the reference's committed run data
 * (notebooks/quick_single_run/data) and the unit known answers of
 * tests/cpp/lennardjonesium; see tests/test_oracle_*.py.
 */

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <thread>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// Pair potentials
// ---------------------------------------------------------------------------

enum ForceKind { FORCE_NONE = 0, FORCE_LJ = 1, FORCE_CONSTANT = 2 };

struct Potential {
    int kind = FORCE_LJ;
    double rc = 2.5;
    double rc2 = 6.25;
    double alpha = 0.0;   // LJ spline constant
    double beta = 0.0;    // LJ spline slope
    double strength = 0.0;  // constant-force mock

    // physics/lennard_jones_force.cpp:33-74 (constructor: spline parameters)
    static Potential lj(double rc) {
        Potential p;
        p.kind = FORCE_LJ;
        p.rc = rc;
        p.rc2 = rc * rc;
        double rcm6 = 1 / (p.rc2 * p.rc2 * p.rc2);
        p.alpha = -4.0 * rcm6 * (rcm6 - 1.0);
        p.beta = 12.0 * rcm6 * (2.0 * rcm6 - 1.0);
        return p;
    }

    // tests/cpp/mock/constant_short_range_force.cpp:31-59 (test mock)
    static Potential constant(double strength, double rc) {
        Potential p;
        p.kind = FORCE_CONSTANT;
        p.rc = rc;
        p.rc2 = rc * rc;
        p.strength = strength;
        return p;
    }

    // Returns true if in range; fills F (3), V, W.
    // LJ: physics/lennard_jones_force.cpp:76-128, arithmetic order of :107-119.
    bool compute(const double s[3], double r2, double F[3], double& V, double& W) const {
        if (kind == FORCE_LJ) {
            if (!(r2 < rc2)) { F[0] = F[1] = F[2] = 0; V = W = 0; return false; }
            double r6 = 1.0 / (r2 * r2 * r2);
            V = 4.0 * r6 * (r6 - 1.0) + alpha + beta * (r2 / rc2 - 1.0);
            W = 24.0 * r6 * (2.0 * r6 - 1.0) - 2.0 * beta * (r2 / rc2);
            for (int k = 0; k < 3; ++k) F[k] = W * s[k] / r2;
            return true;
        }
        if (kind == FORCE_CONSTANT) {
            double norm = std::sqrt(r2);
            if (!(norm < rc)) { F[0] = F[1] = F[2] = 0; V = W = 0; return false; }
            V = strength * (rc - norm);
            W = strength * norm;
            for (int k = 0; k < 3; ++k) F[k] = W * s[k] / (norm * norm);
            return true;
        }
        F[0] = F[1] = F[2] = 0; V = W = 0;
        return false;
    }
};

inline double sq_norm3(const double s[3]) {
    return std::fma(s[2], s[2], std::fma(s[1], s[1], s[0] * s[0]));
}

// ---------------------------------------------------------------------------
// Cell list: tools/cell_list_array.cpp:34-157, engine/particle_pair_filter.cpp:132-192
// ---------------------------------------------------------------------------

struct CellGrid {
    int n[3];
    double ratio[3];  // n_k / L_k (particle_pair_filter.cpp:144-147, ratio first)
    int ncell() const { return n[0] * n[1] * n[2]; }
    int flat(int a, int b, int c) const { return (a * n[1] + b) * n[2] + c; }
};

// tools/cell_list_array.cpp:48 -- shape = floor(L / rc)
CellGrid make_grid(const double L[3], double cell_min) {
    CellGrid g;
    for (int k = 0; k < 3; ++k) {
        g.n[k] = static_cast<int>(std::floor(L[k] / cell_min));
        if (g.n[k] < 1) g.n[k] = 1;
        g.ratio[k] = static_cast<double>(g.n[k]) / L[k];
    }
    return g;
}

inline int cell_coord(double x, double ratio, int n) {
    int c = static_cast<int>(std::floor(x * ratio));
    return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

// Rebinning (particle_pair_filter.cpp:141-154): each cell holds ascending atom ids.
struct Cells {
    CellGrid g;
    std::vector<int> cell_of;   // per atom
    std::vector<int> offsets;   // ncell + 1, exclusive prefix of counts
    std::vector<int> members;   // atom ids, cell-major, ascending within a cell
};

Cells bin_atoms(int N, const double* x, int stride, const CellGrid& g) {
    Cells c;
    c.g = g;
    int nc = g.ncell();
    c.cell_of.resize(N);
    c.offsets.assign(nc + 1, 0);
    for (int i = 0; i < N; ++i) {
        const double* p = x + (size_t)i * stride;
        int a = cell_coord(p[0], g.ratio[0], g.n[0]);
        int b = cell_coord(p[1], g.ratio[1], g.n[1]);
        int d = cell_coord(p[2], g.ratio[2], g.n[2]);
        c.cell_of[i] = g.flat(a, b, d);
        c.offsets[c.cell_of[i] + 1]++;
    }
    for (int k = 0; k < nc; ++k) c.offsets[k + 1] += c.offsets[k];
    c.members.resize(N);
    std::vector<int> fill(c.offsets.begin(), c.offsets.end() - 1);
    for (int i = 0; i < N; ++i) c.members[fill[c.cell_of[i]]++] = i;
    return c;
}

// tools/cell_list_array.cpp:108-114 -- the 13 "positive" neighbour steps
constexpr int kSteps[13][3] = {
    {1, 1, 1}, {1, 1, 0}, {1, 1, -1},
    {1, 0, 1}, {1, 0, 0}, {1, 0, -1},
    {1, -1, 1}, {1, -1, 0}, {1, -1, -1},
    {0, 1, 1}, {0, 1, 0}, {0, 1, -1},
    {0, 0, 1}};

// Enumerate the reference's pair set in the reference's order and call f(i, j, s, r2, img).
// particle_pair_filter.cpp:157-171 (intra-cell i<j), then :174-191 over
// cell_list_array.cpp:118-156 (13 neighbours per cell with lattice image).
template <class Fn>
void for_each_pair_cells(const Cells& c, const double* x, int stride, const double L[3],
                         double rc2, Fn&& f) {
    const CellGrid& g = c.g;
    // 2. intra-cell pairs, cells in x-major order
    for (int cell = 0; cell < g.ncell(); ++cell) {
        int beg = c.offsets[cell], end = c.offsets[cell + 1];
        for (int a = beg; a < end; ++a)
            for (int b = a + 1; b < end; ++b) {
                int i = c.members[a], j = c.members[b];
                const double* pi = x + (size_t)i * stride;
                const double* pj = x + (size_t)j * stride;
                double s[3] = {pi[0] - pj[0], pi[1] - pj[1], pi[2] - pj[2]};
                double r2 = sq_norm3(s);
                if (r2 < rc2) { int img[3] = {0, 0, 0}; f(i, j, s, r2, img); }
            }
    }
    // 3. adjacent cells with lattice image
    for (int ca = 0; ca < g.n[0]; ++ca)
        for (int cb = 0; cb < g.n[1]; ++cb)
            for (int cc = 0; cc < g.n[2]; ++cc) {
                int idx[3] = {ca, cb, cc};
                int first = g.flat(ca, cb, cc);
                for (const auto& st : kSteps) {
                    int nb[3], img[3];
                    for (int k = 0; k < 3; ++k) {
                        nb[k] = idx[k] + st[k];
                        img[k] = (nb[k] < 0 || nb[k] >= g.n[k]) ? st[k] : 0;
                        nb[k] -= img[k] * g.n[k];
                    }
                    int second = g.flat(nb[0], nb[1], nb[2]);
                    double shift[3] = {img[0] * L[0], img[1] * L[1], img[2] * L[2]};
                    for (int a = c.offsets[first]; a < c.offsets[first + 1]; ++a)
                        for (int b = c.offsets[second]; b < c.offsets[second + 1]; ++b) {
                            int i = c.members[a], j = c.members[b];
                            const double* pi = x + (size_t)i * stride;
                            const double* pj = x + (size_t)j * stride;
                            double s[3];
                            for (int k = 0; k < 3; ++k) s[k] = (pi[k] - pj[k]) - shift[k];
                            double r2 = sq_norm3(s);
                            if (r2 < rc2) f(i, j, s, r2, img);
                        }
                }
            }
}

// engine/particle_pair_filter.cpp:68-123 -- naive O(N^2 * 27) filter (test baseline)
template <class Fn>
void for_each_pair_naive(int N, const double* x, int stride, const double L[3], double rc2,
                         Fn&& f) {
    for (int i = 0; i < N; ++i)
        for (int j = i + 1; j < N; ++j)
            for (int a = -1; a <= 1; ++a)
                for (int b = -1; b <= 1; ++b)
                    for (int d = -1; d <= 1; ++d) {
                        int img[3] = {a, b, d};
                        const double* pi = x + (size_t)i * stride;
                        const double* pj = x + (size_t)j * stride;
                        double s[3];
                        for (int k = 0; k < 3; ++k) s[k] = (pi[k] - pj[k]) - img[k] * L[k];
                        double r2 = sq_norm3(s);
                        if (r2 < rc2) f(i, j, s, r2, img);
                    }
}

// ---------------------------------------------------------------------------
// State and the velocity-Verlet step
// ---------------------------------------------------------------------------

struct State {
    int N = 0;
    std::vector<double> x, v, d, F;  // 4 x N, column-major (physics/system_state.hpp:85-95)
    double pe = 0, vir = 0, t = 0;
    explicit State(int n = 0) : N(n), x(4 * (size_t)n, 0.0), v(4 * (size_t)n, 0.0),
                                d(4 * (size_t)n, 0.0), F(4 * (size_t)n, 0.0) {}
};

struct Engine {
    double L[3] = {1, 1, 1};
    double dt = 0.005;
    bool periodic = true;
    Potential pot;
    CellGrid grid;

    // engine/force_calculation.cpp:46-71 (clear_dynamics: physics/system_state.cpp:40-47)
    void forces(State& s) const {
        std::fill(s.F.begin(), s.F.end(), 0.0);
        s.pe = 0;
        s.vir = 0;
        if (pot.kind == FORCE_NONE) return;
        Cells c = bin_atoms(s.N, s.x.data(), 4, grid);
        double* F = s.F.data();
        for_each_pair_cells(c, s.x.data(), 4, L, pot.rc2,
                            [&](int i, int j, const double sep[3], double r2, const int*) {
                                double f[3], V, W;
                                pot.compute(sep, r2, f, V, W);
                                for (int k = 0; k < 3; ++k) {
                                    F[4 * (size_t)i + k] += f[k];
                                    F[4 * (size_t)j + k] -= f[k];
                                }
                                s.pe += V;
                                s.vir += W;
                            });
    }

    // engine/boundary_condition.cpp:37-50 -- x -= floor(x / L) * L
    void wrap(State& s) const {
        for (int i = 0; i < s.N; ++i)
            for (int k = 0; k < 3; ++k) {
                double& x = s.x[4 * (size_t)i + k];
                x -= std::floor(x / L[k]) * L[k];
            }
    }

    // engine/integrator.cpp:62-88 -- one velocity-Verlet step.  A FORCE_NONE
    // potential means "no force calculation" (forces are left as they are), as
    // for an Integrator built without a ShortRangeForce.
    void step(State& s) const {
        size_t n4 = 4 * (size_t)s.N;
        for (size_t q = 0; q < n4; ++q) s.v[q] += (1. / 2.) * s.F[q] * dt;
        for (size_t q = 0; q < n4; ++q) {
            double inc = s.v[q] * dt;
            s.x[q] += inc;
            s.d[q] += inc;
        }
        if (periodic) wrap(s);
        if (pot.kind != FORCE_NONE) forces(s);
        for (size_t q = 0; q < n4; ++q) s.v[q] += (1. / 2.) * s.F[q] * dt;
        s.t += dt;
    }
};

// physics/derived_properties.cpp:37-51 and derived_properties.hpp:75-80
double kinetic_energy(const State& s) {
    double acc = 0;
    for (int i = 0; i < s.N; ++i) {
        const double* v = &s.v[4 * (size_t)i];
        acc += v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    }
    return (1. / 2.) * acc;
}

double mean_square_displacement(const State& s) {
    double acc = 0;
    for (int i = 0; i < s.N; ++i) {
        const double* d = &s.d[4 * (size_t)i];
        acc += d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    }
    return acc / static_cast<double>(s.N);
}

double temperature(const State& s, double ke) { return (2. / 3.) * ke / static_cast<double>(s.N); }

// physics/measurements.hpp:59-70 -- {t, KE, PE, TE, W, T, MSD}
void measure(const State& s, double out[7]) {
    double ke = kinetic_energy(s);
    out[0] = s.t;
    out[1] = ke;
    out[2] = s.pe;
    out[3] = s.pe + ke;
    out[4] = s.vir;
    out[5] = temperature(s, ke);
    out[6] = mean_square_displacement(s);
}

// physics/transformations.cpp:94-116
void set_temperature(State& s, double target) {
    double T = temperature(s, kinetic_energy(s));
    double f = std::sqrt(target / T);
    for (auto& q : s.v) q *= f;
}

// ---------------------------------------------------------------------------
// Initial condition: tools/cubic_lattice.cpp:38-86, engine/initial_condition.cpp:49-104
// ---------------------------------------------------------------------------

struct Lattice {
    int cells_per_side;
    double scale;
    double side() const { return static_cast<double>(cells_per_side) * scale; }
};

Lattice fcc_lattice(int N, double density) {
    Lattice lat;
    int nonempty = static_cast<int>(std::ceil(static_cast<double>(N) / 4.0));
    lat.cells_per_side = static_cast<int>(std::ceil(std::cbrt(static_cast<double>(nonempty))));
    double cps3 = static_cast<double>(lat.cells_per_side * lat.cells_per_side * lat.cells_per_side);
    double proto = static_cast<double>(N) / cps3;
    lat.scale = std::cbrt(proto / density);
    return lat;
}

constexpr double kFcc[4][3] = {{0.0, 0.0, 0.0}, {0.5, 0.5, 0.0}, {0.5, 0.0, 0.5}, {0.0, 0.5, 0.5}};

void lattice_positions(int N, const Lattice& lat, double* x) {
    for (int index = 0; index < N; ++index) {
        auto xyz_s = std::div(index, 4);
        auto xy_z = std::div(xyz_s.quot, lat.cells_per_side);
        auto x_y = std::div(xy_z.quot, lat.cells_per_side);
        int cell[3] = {x_y.quot, x_y.rem, xy_z.rem};
        for (int k = 0; k < 3; ++k)
            x[4 * (size_t)index + k] = (static_cast<double>(cell[k]) + kFcc[xyz_s.rem][k]) * lat.scale;
        x[4 * (size_t)index + 3] = 0.0;
    }
}

// Solve A w = b for a symmetric 3x3 A by Gaussian elimination with partial pivoting.
// (The reference uses Eigen's fullPivHouseholderQr on the 4x4 inertia tensor,
// transformations.cpp:72-73; the 4th row/column decouples, so the 3x3 solve has
// the same solution up to rounding.)
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

void initial_state(int N, double T, double density, unsigned seed, State& s, double& side) {
    s = State(N);
    Lattice lat = fcc_lattice(N, density);
    side = lat.side();
    lattice_positions(N, lat, s.x.data());
    // initial_condition.cpp:76-86 -- component order x0, y0, z0, x1, ...
    std::mt19937 gen{seed};
    std::normal_distribution<> mb{0, std::sqrt(T)};
    for (int i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) s.v[4 * (size_t)i + k] = mb(gen);
    // center of mass before any velocity change (initial_condition.cpp:96)
    double com[3] = {0, 0, 0};
    for (int i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) com[k] += s.x[4 * (size_t)i + k];
    for (int k = 0; k < 3; ++k) com[k] /= static_cast<double>(N);
    // zero momentum (transformations.cpp:35-54)
    double p[3] = {0, 0, 0};
    for (int i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) p[k] += s.v[4 * (size_t)i + k];
    for (int k = 0; k < 3; ++k) {
        double dv = (0.0 - p[k]) / static_cast<double>(N);
        for (int i = 0; i < N; ++i) s.v[4 * (size_t)i + k] += dv;
    }
    // zero angular momentum about the centre of mass (transformations.cpp:56-90)
    double I[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    double Lm[3] = {0, 0, 0};
    for (int i = 0; i < N; ++i) {
        double r[3], v[3];
        for (int k = 0; k < 3; ++k) {
            r[k] = s.x[4 * (size_t)i + k] - com[k];
            v[k] = s.v[4 * (size_t)i + k];
        }
        double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) I[a][b] += (a == b ? r2 : 0.0) - r[a] * r[b];
        Lm[0] += r[1] * v[2] - r[2] * v[1];
        Lm[1] += r[2] * v[0] - r[0] * v[2];
        Lm[2] += r[0] * v[1] - r[1] * v[0];
    }
    double rhs[3] = {-Lm[0], -Lm[1], -Lm[2]};
    double w[3] = {0, 0, 0};
    solve3(I, rhs, w);
    for (int i = 0; i < N; ++i) {
        double r[3];
        for (int k = 0; k < 3; ++k) r[k] = s.x[4 * (size_t)i + k] - com[k];
        s.v[4 * (size_t)i + 0] += w[1] * r[2] - w[2] * r[1];
        s.v[4 * (size_t)i + 1] += w[2] * r[0] - w[0] * r[2];
        s.v[4 * (size_t)i + 2] += w[0] * r[1] - w[1] * r[0];
    }
    set_temperature(s, T);
}

// ---------------------------------------------------------------------------
// Control protocol: control/simulation_controller.cpp:39-146,
// control/simulation_phase.cpp:40-135, physics/analyzers.cpp:44-159,
// tools/moving_sample.hpp:107-188.
// ---------------------------------------------------------------------------

struct Window {
    std::vector<double> buf;
    size_t cap, head = 0, count = 0;
    explicit Window(int n) : buf((size_t)n), cap((size_t)n) {}
    void push(double v) { buf[(head + count) % cap] = v; if (count < cap) ++count; else head = (head + 1) % cap; }
    double at(size_t k) const { return buf[(head + k) % cap]; }
    double mean() const { double a = 0; for (size_t k = 0; k < count; ++k) a += at(k); return a / (double)count; }
    double var() const {
        double m = mean(), a = 0;
        for (size_t k = 0; k < count; ++k) a += (at(k) - m) * (at(k) - m);
        return a / (double)(count - 1);
    }
};

// One ordered pair of the textbook RDF histogram: minimum-image separation
// dd - image * L with image from dd > L/2, r^2 as sq_norm3, bin
// floor(sqrt(r^2) * nbins / rmax).
inline void rdf_count_pair(const double* pi, const double* pj, const double L[3], double rmax2, double inv_dr,
                           int nbins, unsigned long long* hist) {
    double s[3];
    for (int k = 0; k < 3; ++k) {
        double dd = pi[k] - pj[k];
        double img = dd > 0.5 * L[k] ? 1.0 : (dd < -0.5 * L[k] ? -1.0 : 0.0);
        s[k] = dd - img * L[k];
    }
    double r2 = sq_norm3(s);
    if (r2 < rmax2) {
        int b = static_cast<int>(std::sqrt(r2) * inv_dr);
        if (b < nbins) hist[b]++;
    }
}

}  // namespace

// ===========================================================================
// C ABI for ctypes (tests / smoke / CPU baseline only)
// ===========================================================================

extern "C" {

struct ljref_sim_config {
    double temperature, density;
    int particle_count;
    unsigned random_seed;
    double cutoff_distance, time_delta;
    double eq_tolerance;
    int eq_sample_size, eq_adjustment_interval, eq_steady_state_time, eq_timeout;
    double ob_tolerance;
    int ob_sample_size, ob_observation_interval, ob_observation_count;
};

int ljref_version(void) { return 1; }

// Potential value, virial and z-force at a separation along z (forces.hpp:80-84)
int ljref_pair_along_z(int kind, double rc, double strength, double r, double out[3]) {
    Potential p = kind == FORCE_CONSTANT ? Potential::constant(strength, rc) : Potential::lj(rc);
    double s[3] = {0, 0, r};
    double F[3], V, W;
    p.compute(s, sq_norm3(s), F, V, W);
    out[0] = V;
    out[1] = W;
    out[2] = F[2];
    return 0;
}

int ljref_spline(double rc, double out[2]) {
    Potential p = Potential::lj(rc);
    out[0] = p.alpha;
    out[1] = p.beta;
    return 0;
}

// FCC lattice + Maxwell-Boltzmann init; x, v are 4 x N.  Returns the box side in *side.
int ljref_initial_state(int N, double T, double density, unsigned seed, double* x, double* v,
                        double* side) {
    if (N <= 0) return -1;
    State s;
    initial_state(N, T, density, seed, s, *side);
    std::memcpy(x, s.x.data(), sizeof(double) * 4 * (size_t)N);
    std::memcpy(v, s.v.data(), sizeof(double) * 4 * (size_t)N);
    return 0;
}

int ljref_cell_shape(const double L[3], double rc, int shape[3]) {
    CellGrid g = make_grid(L, rc);
    for (int k = 0; k < 3; ++k) shape[k] = g.n[k];
    return 0;
}

// Reference binning: cell_of[N], offsets[ncell+1], members[N] (ascending ids per cell).
int ljref_bin(int N, const double* x, int stride, const double L[3], double rc, int* cell_of,
              int* offsets, int* members) {
    CellGrid g = make_grid(L, rc);
    Cells c = bin_atoms(N, x, stride, g);
    std::memcpy(cell_of, c.cell_of.data(), sizeof(int) * (size_t)N);
    std::memcpy(offsets, c.offsets.data(), sizeof(int) * (size_t)(g.ncell() + 1));
    std::memcpy(members, c.members.data(), sizeof(int) * (size_t)N);
    return g.ncell();
}

// Reference pair set.  mode 0: cell list (reference order), 1: naive.
// Writes up to cap pairs as (i, j, image code) with code = 9*(ix+1)+3*(iy+1)+(iz+1),
// plus r2.  Returns the total number of pairs (may exceed cap).
long long ljref_pairs(int mode, int N, const double* x, int stride, const double L[3], double rc,
                      long long cap, int* pi, int* pj, int* pimg, double* pr2) {
    CellGrid g = make_grid(L, rc);
    long long n = 0;
    auto sink = [&](int i, int j, const double*, double r2, const int* img) {
        if (n < cap) {
            pi[n] = i;
            pj[n] = j;
            pimg[n] = 9 * (img[0] + 1) + 3 * (img[1] + 1) + (img[2] + 1);
            pr2[n] = r2;
        }
        ++n;
    };
    double rc2 = rc * rc;
    if (mode == 0) {
        Cells c = bin_atoms(N, x, stride, g);
        for_each_pair_cells(c, x, stride, L, rc2, sink);
    } else {
        for_each_pair_naive(N, x, stride, L, rc2, sink);
    }
    return n;
}

// One force evaluation (ShortRangeForceCalculation).  x, F are 4 x N.
int ljref_forces(int N, const double* x, const double L[3], int kind, double rc, double strength,
                 double* F, double* pe, double* vir) {
    Engine e;
    for (int k = 0; k < 3; ++k) e.L[k] = L[k];
    e.pot = kind == FORCE_CONSTANT ? Potential::constant(strength, rc) : Potential::lj(rc);
    if (kind == FORCE_NONE) e.pot.kind = FORCE_NONE;
    e.grid = make_grid(L, rc);
    State s(N);
    std::memcpy(s.x.data(), x, sizeof(double) * 4 * (size_t)N);
    e.forces(s);
    std::memcpy(F, s.F.data(), sizeof(double) * 4 * (size_t)N);
    *pe = s.pe;
    *vir = s.vir;
    return 0;
}

// Per-atom sum of |pair force| (for condition-aware force tolerances).
int ljref_force_abs_sum(int N, const double* x, const double L[3], double rc, double* Fabs) {
    Potential p = Potential::lj(rc);
    CellGrid g = make_grid(L, rc);
    Cells c = bin_atoms(N, x, 4, g);
    std::fill(Fabs, Fabs + N, 0.0);
    for_each_pair_cells(c, x, 4, L, p.rc2, [&](int i, int j, const double* s, double r2, const int*) {
        double f[3], V, W;
        p.compute(s, r2, f, V, W);
        double m = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
        Fabs[i] += m;
        Fabs[j] += m;
    });
    return 0;
}

// Advance nsteps of velocity Verlet in place.  x, v, d, F are 4 x N.  thermo
// (7 doubles per step, may be null) receives {t, KE, PE, TE, W, T, MSD}.
// periodic = 0 skips the boundary condition; kind = 0 skips the force calculation.
int ljref_run_steps(int N, double* x, double* v, double* d, double* F, double* t, double* pe,
                    double* vir, const double L[3], double dt, int periodic, int kind, double rc,
                    double strength, int nsteps, double* thermo) {
    Engine e;
    for (int k = 0; k < 3; ++k) e.L[k] = L[k];
    e.dt = dt;
    e.periodic = periodic != 0;
    e.pot = kind == FORCE_CONSTANT ? Potential::constant(strength, rc) : Potential::lj(rc);
    if (kind == FORCE_NONE) e.pot.kind = FORCE_NONE;
    e.grid = make_grid(L, rc);
    State s(N);
    size_t bytes = sizeof(double) * 4 * (size_t)N;
    std::memcpy(s.x.data(), x, bytes);
    std::memcpy(s.v.data(), v, bytes);
    std::memcpy(s.d.data(), d, bytes);
    std::memcpy(s.F.data(), F, bytes);
    s.t = *t;
    s.pe = *pe;
    s.vir = *vir;
    for (int n = 0; n < nsteps; ++n) {
        e.step(s);
        if (thermo) measure(s, thermo + 7 * (size_t)n);
    }
    std::memcpy(x, s.x.data(), bytes);
    std::memcpy(v, s.v.data(), bytes);
    std::memcpy(d, s.d.data(), bytes);
    std::memcpy(F, s.F.data(), bytes);
    *t = s.t;
    *pe = s.pe;
    *vir = s.vir;
    return 0;
}

int ljref_set_temperature(int N, double* v, double target) {
    State s(N);
    std::memcpy(s.v.data(), v, sizeof(double) * 4 * (size_t)N);
    set_temperature(s, target);
    std::memcpy(v, s.v.data(), sizeof(double) * 4 * (size_t)N);
    return 0;
}

// Textbook radial distribution histogram: ordered pairs (i != j) at minimum-image
// distance r < rmax, bin = floor(sqrt(r2) * (nbins / rmax)).  Requires rmax <= L/2.
// (No reference counterpart: the reference has no RDF.)
int ljref_rdf(int N, const double* x, int stride, const double L[3], int nbins, double rmax,
              unsigned long long* hist) {
    std::fill(hist, hist + nbins, 0ULL);
    double rmax2 = rmax * rmax;
    double inv_dr = static_cast<double>(nbins) / rmax;
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            if (i == j) continue;
            rdf_count_pair(x + (size_t)i * stride, x + (size_t)j * stride, L, rmax2, inv_dr, nbins, hist);
        }
    return 0;
}

// The same histogram as ljref_rdf for large systems: the candidates of atom i
// are the atoms of the 27 cells around its own on a grid of cells of edge
// >= rmax (at least 3 per axis, so the 27 cells are distinct and hold every
// atom within rmax); each ordered pair gets exactly ljref_rdf's arithmetic.
// Atom ranges run on `threads` host threads with private histograms summed at
// the end (integer counts: the sum is order-free).  Returns 1 if the box is
// under 3 cells of edge rmax per axis.
int ljref_rdf_cells(int N, const double* x, int stride, const double L[3], int nbins, double rmax,
                    int threads, unsigned long long* hist) {
    CellGrid g = make_grid(L, rmax);
    if (g.n[0] < 3 || g.n[1] < 3 || g.n[2] < 3) return 1;
    Cells c = bin_atoms(N, x, stride, g);
    double rmax2 = rmax * rmax;
    double inv_dr = static_cast<double>(nbins) / rmax;
    if (threads < 1) threads = 1;
    std::vector<std::vector<unsigned long long>> part(threads, std::vector<unsigned long long>(nbins, 0ULL));
    auto work = [&](int t) {
        unsigned long long* h = part[t].data();
        for (int i = t; i < N; i += threads) {
            int ci = c.cell_of[i];
            int a = ci / (g.n[1] * g.n[2]), b = (ci / g.n[2]) % g.n[1], d = ci % g.n[2];
            for (int da = -1; da <= 1; ++da)
                for (int db = -1; db <= 1; ++db)
                    for (int dd = -1; dd <= 1; ++dd) {
                        int cell = g.flat((a + da + g.n[0]) % g.n[0], (b + db + g.n[1]) % g.n[1],
                                          (d + dd + g.n[2]) % g.n[2]);
                        for (int k = c.offsets[cell]; k < c.offsets[cell + 1]; ++k) {
                            int j = c.members[k];
                            if (j == i) continue;
                            rdf_count_pair(x + (size_t)i * stride, x + (size_t)j * stride, L, rmax2, inv_dr,
                                           nbins, h);
                        }
                    }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    std::fill(hist, hist + nbins, 0ULL);
    for (int t = 0; t < threads; ++t)
        for (int b = 0; b < nbins; ++b) hist[b] += part[t][b];
    return 0;
}

// Full simulation with the reference's control protocol, writing the per-step
// thermodynamic records (7 doubles each) into thermo (capacity max_steps) and
// the event list as text into events (capacity events_cap bytes).  Returns the
// number of steps taken, or -1 if thermo was too small.
long long ljref_simulate(const ljref_sim_config* cfg, long long max_steps, double* thermo,
                         char* events, int events_cap, double* snapshot_xvf) {
    State s;
    double side;
    initial_state(cfg->particle_count, cfg->temperature, cfg->density, cfg->random_seed, s, side);
    Engine e;
    e.L[0] = e.L[1] = e.L[2] = side;
    e.dt = cfg->time_delta;
    e.pot = Potential::lj(cfg->cutoff_distance);
    e.grid = make_grid(e.L, cfg->cutoff_distance);
    std::string ev;
    auto log = [&](int step, const std::string& msg) { ev += std::to_string(step) + ": " + msg + "\n"; };
    char buf[256];
    int time_step = 0;
    long long nrec = 0;
    int N = cfg->particle_count;
    double rho = cfg->density;
    for (int phase = 0; phase < 2; ++phase) {
        bool eq = phase == 0;
        log(time_step, std::string("Phase started: ") + (eq ? "Equilibration Phase" : "Observation Phase"));
        int start = time_step, last_check = time_step, last_adjust = time_step, last_obs = time_step;
        int nobs = 0;
        Window Tw(eq ? cfg->eq_sample_size : cfg->ob_sample_size);
        Window Ew(cfg->ob_sample_size), Ww(cfg->ob_sample_size);
        Window tw(cfg->ob_sample_size), mw(cfg->ob_sample_size);
        bool done = false, aborted = false;
        while (!done) {
            e.step(s);
            if (nrec >= max_steps) return -1;
            double* rec = thermo + 7 * (size_t)nrec++;
            measure(s, rec);
            time_step += 1;
            if (eq) {
                Tw.push(rec[5]);
                if (time_step - last_check >= cfg->eq_adjustment_interval) {
                    last_check = time_step;
                    double Tm = Tw.mean();
                    if (std::fabs(Tm / cfg->temperature - 1.0) >= cfg->eq_tolerance) {
                        last_adjust = time_step;
                        std::snprintf(buf, sizeof buf, "Temperature measured at: %.4g, adjusted to: %.4g",
                                      Tm, cfg->temperature);
                        log(time_step, buf);
                        set_temperature(s, cfg->temperature);
                    }
                }
                if (time_step - last_adjust >= cfg->eq_steady_state_time) {
                    log(time_step, "Phase complete: Equilibration Phase");
                    done = true;
                } else if (time_step - start >= cfg->eq_timeout) {
                    log(time_step, "Simulation aborted: Could not equilibrate");
                    done = aborted = true;
                }
            } else {
                Tw.push(rec[5]);
                Ew.push(rec[3]);
                Ww.push(rec[4]);
                tw.push(rec[0]);
                mw.push(rec[6]);
                if (time_step - last_obs >= cfg->ob_observation_interval) {
                    last_obs = time_step;
                    double Tm = Tw.mean();
                    if (std::fabs(Tm / cfg->temperature - 1.0) >= cfg->ob_tolerance) {
                        log(time_step, "Simulation aborted: Temperature drifted outside acceptable range");
                        done = aborted = true;
                        continue;
                    }
                    ++nobs;
                    log(time_step, "Observation recorded");
                    (void)rho;
                }
                if (nobs >= cfg->ob_observation_count) {
                    log(time_step, "Phase complete: Observation Phase");
                    done = true;
                }
            }
        }
        if (aborted) break;
    }
    if (events && events_cap > 0) {
        std::snprintf(events, (size_t)events_cap, "%s", ev.c_str());
    }
    if (snapshot_xvf) {
        for (int i = 0; i < N; ++i)
            for (int k = 0; k < 3; ++k) {
                snapshot_xvf[9 * (size_t)i + k] = s.x[4 * (size_t)i + k];
                snapshot_xvf[9 * (size_t)i + 3 + k] = s.v[4 * (size_t)i + k];
                snapshot_xvf[9 * (size_t)i + 6 + k] = s.F[4 * (size_t)i + k];
            }
    }
    return nrec;
}

// CPU baseline: run `replicas` independent copies of an FCC system on as many
// threads (the reference's SimulationPool parallelism, api/simulation_pool.cpp:35-42),
// each doing warm + steps velocity-Verlet steps with per-step measurement.
// Returns the wall seconds of the timed steps (max over threads) in *seconds.
int ljref_bench(int N, double T, double density, unsigned seed, double rc, double dt, int warm,
                int steps, int replicas, double* seconds) {
    std::vector<double> secs((size_t)replicas, 0.0);
    std::vector<std::thread> pool;
    std::atomic<int> ready{0};
    for (int r = 0; r < replicas; ++r) {
        pool.emplace_back([&, r]() {
            State s;
            double side;
            initial_state(N, T, density, seed + (unsigned)r, s, side);
            Engine e;
            e.L[0] = e.L[1] = e.L[2] = side;
            e.dt = dt;
            e.pot = Potential::lj(rc);
            e.grid = make_grid(e.L, rc);
            double rec[7];
            for (int n = 0; n < warm; ++n) { e.step(s); measure(s, rec); }
            ready.fetch_add(1);
            while (ready.load() < replicas) std::this_thread::yield();
            timespec a, b;
            clock_gettime(CLOCK_MONOTONIC, &a);
            for (int n = 0; n < steps; ++n) { e.step(s); measure(s, rec); }
            clock_gettime(CLOCK_MONOTONIC, &b);
            secs[(size_t)r] = (double)(b.tv_sec - a.tv_sec) + 1e-9 * (double)(b.tv_nsec - a.tv_nsec);
        });
    }
    for (auto& th : pool) th.join();
    *seconds = *std::max_element(secs.begin(), secs.end());
    return 0;
}

}  // extern "C"
