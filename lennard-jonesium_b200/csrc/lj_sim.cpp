// lj_sim.cpp -- host side of a whole simulation over the engine ABI:
// api::Simulation::run (api/simulation.cpp:72-117) with the control protocol of
// control::SimulationController (control/simulation_controller.cpp:39-146), the
// equilibration / observation phases (control/simulation_phase.cpp:40-135), the
// analyzers (physics/analyzers.cpp:44-159, tools/moving_sample.hpp:107-188) and
// the four output sinks (output/sinks.cpp:40-204).
//
// The controller needs, per step, only the 7-scalar ThermodynamicMeasurement;
// a phase can change anything (rescale velocities, record, finish, abort) only
// at steps fixed by its counters (next adjustment check, steady-state and
// timeout deadlines, next observation).  So the GPU runs chunks of steps that
// end exactly at the next such step, the host replays the records through the
// phase logic one step at a time, and the only state mutation
// (set_temperature) happens where the reference does it.

#include <algorithm>
#include <array>
#include <charconv>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <functional>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lj_gpu.h"

namespace {

// fmt's "{}" for a double: the shortest digits that round-trip, fixed notation
// when the decimal exponent is in [-4, 16), scientific ("1e-05") otherwise, no
// trailing ".0" for whole numbers.  Writes at most 32 bytes to out and returns
// the length.
int fmt_double_buf(double v, char* out) {
    char* o = out;
    if (std::isnan(v)) return (int)(std::memcpy(out, "nan", 3), 3);
    if (std::isinf(v)) {
        if (v < 0) *o++ = '-';
        std::memcpy(o, "inf", 3);
        return (int)(o - out) + 3;
    }
    if (v == 0) {
        if (std::signbit(v)) *o++ = '-';
        *o++ = '0';
        return (int)(o - out);
    }
    char buf[40];
    auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::scientific);
    const char* p = buf;
    if (*p == '-') {
        *o++ = '-';
        ++p;
    }
    char digits[24];
    int nd = 0;
    for (; p < r.ptr && *p != 'e'; ++p)
        if (*p != '.') digits[nd++] = *p;
    ++p;  // 'e'
    bool eneg = *p == '-';
    if (*p == '-' || *p == '+') ++p;
    int exp = 0;
    for (; p < r.ptr; ++p) exp = exp * 10 + (*p - '0');
    if (eneg) exp = -exp;
    if (exp >= -4 && exp < 16) {
        if (exp < 0) {
            *o++ = '0';
            *o++ = '.';
            for (int k = 0; k < -exp - 1; ++k) *o++ = '0';
            for (int k = 0; k < nd; ++k) *o++ = digits[k];
        } else if (nd <= exp + 1) {
            for (int k = 0; k < nd; ++k) *o++ = digits[k];
            for (int k = nd; k < exp + 1; ++k) *o++ = '0';
        } else {
            for (int k = 0; k <= exp; ++k) *o++ = digits[k];
            *o++ = '.';
            for (int k = exp + 1; k < nd; ++k) *o++ = digits[k];
        }
    } else {
        *o++ = digits[0];
        if (nd > 1) {
            *o++ = '.';
            for (int k = 1; k < nd; ++k) *o++ = digits[k];
        }
        *o++ = 'e';
        *o++ = exp < 0 ? '-' : '+';
        int a = exp < 0 ? -exp : exp;
        if (a >= 100) *o++ = (char)('0' + a / 100);
        *o++ = (char)('0' + (a / 10) % 10);
        *o++ = (char)('0' + a % 10);
    }
    return (int)(o - out);
}

std::string fmt_double(double v) {
    char b[40];
    return std::string(b, (size_t)fmt_double_buf(v, b));
}

// One thermodynamics.csv row (output/sinks.cpp:116-130) into out (>= 320 bytes).
int thermo_line(int step, const lj_thermo& r, char* out) {
    char* o = out;
    o = std::to_chars(o, o + 16, step).ptr;
    for (double x : {r.time, r.kinetic_energy, r.potential_energy, r.total_energy, r.virial, r.temperature,
                     r.mean_square_displacement}) {
        *o++ = ',';
        o += fmt_double_buf(x, o);
    }
    *o++ = '\n';
    return (int)(o - out);
}

// Writes thermodynamics rows on a background thread, in the order they were
// queued, so that formatting the rows of one chunk of steps overlaps the GPU's
// next chunk.  drain() returns once every queued row is written.
class ThermoWriter {
  public:
    struct Row {
        FILE* f;
        int step;
        lj_thermo r;
    };
    ThermoWriter() : th_([this] { run(); }) {}
    ~ThermoWriter() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
        }
        cv_.notify_all();
        th_.join();
    }
    void push(std::vector<Row>&& rows) {
        if (rows.empty()) return;
        {
            std::lock_guard<std::mutex> g(m_);
            q_.push_back(std::move(rows));
        }
        cv_.notify_all();
    }
    void drain() {
        std::unique_lock<std::mutex> g(m_);
        idle_cv_.wait(g, [this] { return q_.empty() && !busy_; });
    }

  private:
    void run() {
        char line[320];
        for (;;) {
            std::vector<Row> job;
            {
                std::unique_lock<std::mutex> g(m_);
                cv_.wait(g, [this] { return stop_ || !q_.empty(); });
                if (q_.empty()) return;  // stop requested and nothing left
                job = std::move(q_.front());
                q_.pop_front();
                busy_ = true;
            }
            for (const Row& row : job) std::fwrite(line, 1, (size_t)thermo_line(row.step, row.r, line), row.f);
            {
                std::lock_guard<std::mutex> g(m_);
                busy_ = false;
            }
            idle_cv_.notify_all();
        }
    }
    std::mutex m_;
    std::condition_variable cv_, idle_cv_;
    std::deque<std::vector<Row>> q_;
    bool stop_ = false, busy_ = false;
    std::thread th_;
};

// fmt's "{:.4g}"
std::string fmt_g4(double v) {
    char b[64];
    std::snprintf(b, sizeof b, "%.4g", v);
    return b;
}

// std::reduce / std::transform_reduce over a random-access range as libstdc++
// evaluates them (blocks of four, then the tail), for window statistics.
template <class T, class F>
T blocked_sum(const std::vector<T>& xs, T init, F f) {
    size_t n = xs.size(), k = 0;
    for (; n - k >= 4; k += 4) {
        T v1 = f(xs[k]) + f(xs[k + 1]);
        T v2 = f(xs[k + 2]) + f(xs[k + 3]);
        init = init + (v1 + v2);
    }
    for (; k < n; ++k) init = init + f(xs[k]);
    return init;
}

// tools::MovingSample: the last `cap` values, oldest first.
struct Window {
    size_t cap;
    std::vector<double> buf;
    explicit Window(int n) : cap((size_t)n) {}
    void push(double v) {
        buf.push_back(v);
        if (buf.size() > cap) buf.erase(buf.begin());
    }
    double mean() const { return blocked_sum(buf, 0.0, [](double x) { return x; }) / (double)buf.size(); }
    double variance() const {
        double m = mean();
        return blocked_sum(buf, 0.0, [m](double x) { return (x - m) * (x - m); }) / (double)(buf.size() - 1);
    }
};

struct Observation {
    double temperature, density, total_energy, pressure, specific_heat, diffusion_coefficient;
};

struct Sinks {
    FILE* events = nullptr;
    FILE* thermo = nullptr;
    FILE* obs = nullptr;
    FILE* snap = nullptr;
    int echo = 0;
    void event(int step, const std::string& msg) {
        std::string line = std::to_string(step) + ": " + msg + "\n";
        std::fputs(line.c_str(), events);
        std::fflush(events);
        if (echo) {
            std::fputs(line.c_str(), stdout);
            std::fflush(stdout);
        }
    }
    std::vector<ThermoWriter::Row>* pending = nullptr;  // rows for a ThermoWriter, if one is attached
    void thermo_row(int step, const lj_thermo& r) {
        if (pending) {
            pending->push_back({thermo, step, r});
            return;
        }
        char line[320];
        std::fwrite(line, 1, (size_t)thermo_line(step, r, line), thermo);
    }
    void obs_row(int step, const Observation& o) {
        std::string s = std::to_string(step) + "," + fmt_double(o.temperature) + "," + fmt_double(o.density) + "," +
                        fmt_double(o.total_energy) + "," + fmt_double(o.pressure) + "," +
                        fmt_double(o.specific_heat) + "," + fmt_double(o.diffusion_coefficient) + "\n";
        std::fputs(s.c_str(), obs);
    }
    void close() {
        for (FILE* f : {events, thermo, obs, snap})
            if (f) std::fclose(f);
    }
};

// physics::ThermodynamicAnalyzer::result (analyzers.cpp:44-159)
Observation analyze(const Window& T, const Window& E, const Window& W, const Window& t, const Window& msd, int N,
                    double density) {
    Observation o;
    o.temperature = T.mean();
    o.density = density;
    o.total_energy = E.mean();
    o.pressure = density * (o.temperature + W.mean() / (3.0 * N));
    double rtf = T.variance() / (o.temperature * o.temperature);
    o.specific_heat = (3. / 2.) / (1 - (3. / 2.) * N * rtf);
    // Cov(t, msd) / Var(t) over the window (the Bessel factors cancel)
    double tm = t.mean(), mm = msd.mean();
    double ctm = 0, ctt = 0;
    {
        size_t n = t.buf.size(), k = 0;
        double c1 = 0, c0 = 0;
        auto f01 = [&](size_t q) { return (t.buf[q] - tm) * (msd.buf[q] - mm); };
        auto f00 = [&](size_t q) { return (t.buf[q] - tm) * (t.buf[q] - tm); };
        for (; n - k >= 4; k += 4) {
            c1 = c1 + ((f01(k) + f01(k + 1)) + (f01(k + 2) + f01(k + 3)));
            c0 = c0 + ((f00(k) + f00(k + 1)) + (f00(k + 2) + f00(k + 3)));
        }
        for (; k < n; ++k) {
            c1 = c1 + f01(k);
            c0 = c0 + f00(k);
        }
        ctm = c1 / (double)(n - 1);
        ctt = c0 / (double)(n - 1);
    }
    o.diffusion_coefficient = (1. / 6.) * (ctm / ctt);
    return o;
}

double relative_error(double measured, double desired) { return std::abs(measured / desired - 1.0); }

}  // namespace

namespace ljb {

// Rows of the snapshot file (output/sinks.cpp:185-204): "step,id,x,y,z,vx,vy,vz,fx,fy,fz"
// for atoms 0..n-1 of xvf (9 doubles per atom).  Large frames are formatted in
// blocks of kSnapshotBlock rows on up to 16 threads at a time and written in
// row order (a 256 000-atom frame is ~50 MB of text; one thread formats ~2 M
// rows per second).  Returns 0, or 1 if a write failed.
constexpr int kSnapshotBlock = 32768;

static void format_snapshot_block(long long time_step, const double* xvf, int lo, int hi, std::vector<char>& buf) {
    buf.clear();
    char line[400];
    for (int i = lo; i < hi; ++i) {
        char* o = line;
        o = std::to_chars(o, o + 24, time_step).ptr;
        *o++ = ',';
        o = std::to_chars(o, o + 16, i).ptr;
        for (int k = 0; k < 9; ++k) {
            *o++ = ',';
            o += fmt_double_buf(xvf[9 * (size_t)i + k], o);
        }
        *o++ = '\n';
        buf.insert(buf.end(), line, o);
    }
}

int write_snapshot_rows(long long time_step, const double* xvf, int n, FILE* f) {
    unsigned hw = std::thread::hardware_concurrency();
    int P = (int)std::min(16u, std::max(1u, hw));
    std::vector<std::vector<char>> bufs((size_t)P);
    for (int base = 0; base < n; base += P * kSnapshotBlock) {
        int nb = std::min(P, (n - base + kSnapshotBlock - 1) / kSnapshotBlock);
        std::vector<std::thread> th;
        for (int b = 1; b < nb; ++b) {
            int lo = base + b * kSnapshotBlock, hi = std::min(n, lo + kSnapshotBlock);
            th.emplace_back(format_snapshot_block, time_step, xvf, lo, hi, std::ref(bufs[(size_t)b]));
        }
        format_snapshot_block(time_step, xvf, base, std::min(n, base + kSnapshotBlock), bufs[0]);
        for (std::thread& t : th) t.join();
        for (int b = 0; b < nb; ++b) {
            const std::vector<char>& q = bufs[(size_t)b];
            if (!q.empty() && std::fwrite(q.data(), 1, q.size(), f) != q.size()) return 1;
        }
    }
    return std::fflush(f) == 0 ? 0 : 1;
}

}  // namespace ljb

extern "C" {

int lj_window_stats_host(const lj_thermo* records, int n, int particle_count, double density, lj_observation* out) {
    if (!records || !out || n < 2 || particle_count < 1) return LJ_ERR_ARG;
    Window T(n), E(n), W(n), t(n), msd(n);
    for (int k = 0; k < n; ++k) {
        const lj_thermo& r = records[k];
        T.push(r.temperature);
        E.push(r.total_energy);
        W.push(r.virial);
        t.push(r.time);
        msd.push(r.mean_square_displacement);
    }
    Observation o = analyze(T, E, W, t, msd, particle_count, density);
    *out = lj_observation{o.temperature, o.density, o.total_energy, o.pressure, o.specific_heat,
                          o.diffusion_coefficient};
    return LJ_OK;
}

int lj_format_double(double v, char* out, int cap) {
    if (!out || cap < 1) return LJ_ERR_ARG;
    std::string s = fmt_double(v);
    if ((int)s.size() >= cap) return LJ_ERR_ARG;
    std::memcpy(out, s.c_str(), s.size() + 1);
    return LJ_OK;
}

// physics::LennardJonesForce::compute along z (lennard_jones_force.cpp:76-128):
// out = {potential, virial, z-force} at separation r.
int lj_pair_along_z(double cutoff, double r, double* out) {
    if (!out || !(cutoff > 0)) return LJ_ERR_ARG;
    double rc2 = cutoff * cutoff;
    double rcm6 = 1 / (rc2 * rc2 * rc2);
    double alpha = -4.0 * rcm6 * (rcm6 - 1.0), beta = 12.0 * rcm6 * (2.0 * rcm6 - 1.0);
    double r2 = r * r;
    if (!(r2 < rc2)) {
        out[0] = out[1] = out[2] = 0.0;
        return LJ_OK;
    }
    double r6 = 1.0 / (r2 * r2 * r2);
    out[0] = 4.0 * r6 * (r6 - 1.0) + alpha + beta * (r2 / rc2 - 1.0);
    out[1] = 24.0 * r6 * (2.0 * r6 - 1.0) - 2.0 * beta * (r2 / rc2);
    out[2] = out[1] * r / r2;
    return LJ_OK;
}


// The control protocol of one simulation, fed one ThermodynamicMeasurement per
// step.  next_decision() is the first step at which the current phase can act;
// feed() replays a step's record and reports what the controller asks of the
// engine (a velocity rescale) and whether the run has finished.
struct Controller {
    const lj_sim_config* cfg;
    Sinks out;
    int N;
    int time_step = 0;
    int phase = 0;  // 0 equilibration, 1 observation, 2 finished
    int start = 0, last_check = 0, last_adjust = 0, last_obs = 0, count = 0;
    int outcome = 0, nobs = 0;
    Window Tw, Ew, Ww, tw, mw;
    const char* names[2];

    explicit Controller(const lj_sim_config* c)
        : cfg(c), N(c->particle_count), Tw(c->eq_sample_size), Ew(c->ob_sample_size), Ww(c->ob_sample_size),
          tw(c->ob_sample_size), mw(c->ob_sample_size) {
        names[0] = c->eq_name ? c->eq_name : "Equilibration Phase";
        names[1] = c->ob_name ? c->ob_name : "Observation Phase";
    }

    int open(int echo) {
        out.echo = echo;
        out.events = std::fopen(cfg->event_log, "w");
        out.thermo = std::fopen(cfg->thermodynamic_log, "w");
        out.obs = std::fopen(cfg->observation_log, "w");
        out.snap = std::fopen(cfg->snapshot_log, "w");
        if (!out.events || !out.thermo || !out.obs || !out.snap) return LJ_ERR_ARG;
        std::fputs("TimeStep,Time,KineticEnergy,PotentialEnergy,TotalEnergy,Virial,Temperature,"
                   "MeanSquareDisplacement\n", out.thermo);
        std::fputs("TimeStep,Temperature,Density,TotalEnergy,Pressure,SpecificHeat,DiffusionCoefficient\n", out.obs);
        std::fputs("TimeStep,ParticleID,Position,Position,Position,Velocity,Velocity,Velocity,Force,Force,Force\n",
                   out.snap);
        std::fputs("TimeStep,ParticleID,X,Y,Z,X,Y,Z,X,Y,Z\n", out.snap);
        begin_phase();
        return LJ_OK;
    }

    void begin_phase() {
        out.event(time_step, std::string("Phase started: ") + names[phase]);
        start = last_check = last_adjust = last_obs = time_step;
        count = 0;
        Tw = Window(phase == 0 ? cfg->eq_sample_size : cfg->ob_sample_size);
        Ew = Window(cfg->ob_sample_size);
        Ww = Window(cfg->ob_sample_size);
        tw = Window(cfg->ob_sample_size);
        mw = Window(cfg->ob_sample_size);
    }

    bool finished() const { return phase == 2; }

    int next_decision() const {
        if (phase == 0)
            return std::min({last_check + cfg->eq_adjustment_interval, last_adjust + cfg->eq_steady_state_time,
                             start + cfg->eq_timeout});
        return last_obs + cfg->ob_observation_interval;
    }

    // One step's record.  Returns true when the engine must rescale velocities
    // to cfg->temperature before the next step.
    bool feed(const lj_thermo& r) {
        bool rescale = false;
        out.thermo_row(time_step, r);  // logged before the increment (simulation_controller.cpp:65-67)
        time_step += 1;
        if (phase == 0) {
            Tw.push(r.temperature);
            if (time_step - last_check >= cfg->eq_adjustment_interval) {
                last_check = time_step;
                double Tm = Tw.mean();
                if (relative_error(Tm, cfg->temperature) >= cfg->eq_tolerance) {
                    last_adjust = time_step;
                    rescale = true;
                    out.event(time_step, "Temperature measured at: " + fmt_g4(Tm) +
                                             ", adjusted to: " + fmt_g4(cfg->temperature));
                }
            }
            if (time_step - last_adjust >= cfg->eq_steady_state_time) {
                out.event(time_step, std::string("Phase complete: ") + names[0]);
                phase = 1;
                begin_phase();
            } else if (time_step - start >= cfg->eq_timeout) {
                out.event(time_step, "Simulation aborted: Could not equilibrate");
                phase = 2;
                outcome = 1;
            }
        } else if (phase == 1) {
            Tw.push(r.temperature);
            Ew.push(r.total_energy);
            Ww.push(r.virial);
            tw.push(r.time);
            mw.push(r.mean_square_displacement);
            if (time_step - last_obs >= cfg->ob_observation_interval) {
                last_obs = time_step;
                Observation o = analyze(Tw, Ew, Ww, tw, mw, N, cfg->density);
                if (relative_error(o.temperature, cfg->temperature) >= cfg->ob_tolerance) {
                    out.event(time_step, "Simulation aborted: Temperature drifted outside acceptable range");
                    phase = 2;
                    outcome = 2;
                    return false;
                }
                ++count;
                ++nobs;
                out.obs_row(time_step, o);
                out.event(time_step, "Observation recorded");
            }
            if (count >= cfg->ob_observation_count) {
                out.event(time_step, std::string("Phase complete: ") + names[1]);
                phase = 2;
            }
        }
        return rescale;
    }

    // snapshot of the final (or aborted) state (simulation_controller.cpp:100-108, :128-134)
    void snapshot(const double* x, const double* v, const double* F) {
        std::string step = std::to_string(time_step) + ",";
        std::string line;
        for (int i = 0; i < N; ++i) {
            line = step + std::to_string(i);
            for (const double* a : {x, v, F})
                for (int k = 0; k < 3; ++k) line += "," + fmt_double(a[4 * (size_t)i + k]);
            line += "\n";
            std::fputs(line.c_str(), out.snap);
        }
    }
};

int lj_sim_run(const lj_sim_config* cfg, int echo, lj_sim_result* result) {
    if (!cfg || cfg->particle_count < 1 || !cfg->event_log || !cfg->thermodynamic_log || !cfg->observation_log ||
        !cfg->snapshot_log)
        return LJ_ERR_ARG;
    auto t0 = std::chrono::steady_clock::now();
    const int N = cfg->particle_count;
    std::vector<double> x(4 * (size_t)N), v(4 * (size_t)N);
    double side = 0;
    int rc = lj_initial_condition(N, cfg->temperature, cfg->density, cfg->random_seed, x.data(), v.data(), &side);
    if (rc) return rc;
    lj_params p;
    lj_gpu_default_params(&p);
    p.particle_count = N;
    p.box[0] = p.box[1] = p.box[2] = side;
    p.cutoff_distance = cfg->cutoff_distance;
    p.time_delta = cfg->time_delta;
    p.precision = cfg->precision;
    p.device = cfg->device;
    lj_ctx* ctx = nullptr;
    if ((rc = lj_gpu_create(&p, &ctx))) return rc;
    Controller ctl(cfg);
    if ((rc = lj_gpu_upload_state(ctx, x.data(), v.data(), nullptr, nullptr, 4, 0.0, 0.0, 0.0)) ||
        (rc = ctl.open(echo))) {
        ctl.out.close();
        lj_gpu_destroy(ctx);
        return rc;
    }
    std::vector<lj_thermo> recs;
    ThermoWriter writer;
    std::vector<ThermoWriter::Row> rows;
    ctl.out.pending = &rows;
    while (!ctl.finished() && rc == LJ_OK) {
        int K = std::max(1, ctl.next_decision() - ctl.time_step);
        recs.resize((size_t)K);
        if ((rc = lj_gpu_step(ctx, K, recs.data()))) break;
        for (int k = 0; k < K && !ctl.finished(); ++k)
            if (ctl.feed(recs[(size_t)k]) && (rc = lj_gpu_set_temperature(ctx, cfg->temperature, nullptr))) break;
        writer.push(std::move(rows));  // formatted while the GPU runs the next chunk
        rows.clear();
    }
    writer.drain();
    if (rc == LJ_OK) {
        std::vector<double> F(4 * (size_t)N);
        rc = lj_gpu_download_state(ctx, x.data(), v.data(), nullptr, F.data(), 4, nullptr, nullptr, nullptr);
        if (rc == LJ_OK) ctl.snapshot(x.data(), v.data(), F.data());
    }
    ctl.out.close();
    lj_gpu_destroy(ctx);
    if (result) {
        result->time_steps = ctl.time_step;
        result->outcome = ctl.outcome;
        result->observations = ctl.nobs;
        result->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    return rc;
}

// A whole sweep on one batched engine: every configuration's control protocol
// runs on the host as in lj_sim_run, all systems step together, and each chunk
// ends at the earliest step at which any running simulation can act.  The
// configurations must share cutoff and time step.
int lj_sim_run_batch(const lj_sim_config* cfgs, int n, int echo, lj_sim_result* results) {
    if (!cfgs || n < 1) return LJ_ERR_ARG;
    auto t0 = std::chrono::steady_clock::now();
    std::vector<lj_batch_system> systems((size_t)n);
    std::vector<std::vector<double>> xs((size_t)n), vs((size_t)n);
    for (int s = 0; s < n; ++s) {
        const lj_sim_config& c = cfgs[s];
        if (c.particle_count < 1 || c.cutoff_distance != cfgs[0].cutoff_distance ||
            c.time_delta != cfgs[0].time_delta)
            return LJ_ERR_ARG;
        xs[(size_t)s].resize(4 * (size_t)c.particle_count);
        vs[(size_t)s].resize(4 * (size_t)c.particle_count);
        double side = 0;
        int rc = lj_initial_condition(c.particle_count, c.temperature, c.density, c.random_seed,
                                      xs[(size_t)s].data(), vs[(size_t)s].data(), &side);
        if (rc) return rc;
        systems[(size_t)s].particle_count = c.particle_count;
        systems[(size_t)s].box[0] = systems[(size_t)s].box[1] = systems[(size_t)s].box[2] = side;
        systems[(size_t)s].time_delta = c.time_delta;
        systems[(size_t)s].skin = -1.0;
    }
    lj_batch* b = nullptr;
    int rc = lj_batch_create(systems.data(), n, cfgs[0].cutoff_distance, cfgs[0].device, &b);
    if (rc) return rc;
    std::vector<Controller> ctl;
    ctl.reserve((size_t)n);
    for (int s = 0; s < n; ++s) ctl.emplace_back(&cfgs[s]);
    for (int s = 0; s < n && rc == LJ_OK; ++s) {
        rc = lj_batch_upload_system(b, s, xs[(size_t)s].data(), vs[(size_t)s].data(), 4);
        if (rc == LJ_OK) rc = ctl[(size_t)s].open(echo);
    }
    std::vector<lj_thermo> recs;
    ThermoWriter writer;
    std::vector<ThermoWriter::Row> rows;
    for (auto& c : ctl) c.out.pending = &rows;
    int running = n;
    while (running > 0 && rc == LJ_OK) {
        int K = 1 << 30;
        for (auto& c : ctl)
            if (!c.finished()) K = std::min(K, c.next_decision() - c.time_step);
        K = std::max(1, K);
        recs.resize((size_t)K * n);
        if ((rc = lj_batch_step(b, K, recs.data()))) break;
        for (int s = 0; s < n && rc == LJ_OK; ++s) {
            Controller& c = ctl[(size_t)s];
            if (c.finished()) continue;
            bool rescale = false;
            for (int k = 0; k < K && !c.finished(); ++k) rescale = c.feed(recs[(size_t)k * n + s]) || rescale;
            // a rescale precedes an abort on the same step, as in the reference's command queue
            if (rescale) rc = lj_batch_set_temperature(b, s, cfgs[s].temperature, nullptr);
            if (rc == LJ_OK && c.finished()) {
                writer.push(std::move(rows));  // this run's rows before its snapshot
                rows.clear();
                writer.drain();
                const int N = cfgs[s].particle_count;
                std::vector<double> F(4 * (size_t)N);
                rc = lj_batch_download_system(b, s, xs[(size_t)s].data(), vs[(size_t)s].data(), F.data(), 4);
                if (rc == LJ_OK) c.snapshot(xs[(size_t)s].data(), vs[(size_t)s].data(), F.data());
                if (rc == LJ_OK) rc = lj_batch_set_active(b, s, 0);
                --running;
            }
        }
        writer.push(std::move(rows));  // formatted while the GPU runs the next chunk
        rows.clear();
    }
    writer.drain();
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int s = 0; s < n; ++s) {
        ctl[(size_t)s].out.close();
        if (results) {
            results[s].time_steps = ctl[(size_t)s].time_step;
            results[s].outcome = ctl[(size_t)s].outcome;
            results[s].observations = ctl[(size_t)s].nobs;
            results[s].seconds = secs;
        }
    }
    lj_batch_destroy(b);
    return rc;
}

}  // extern "C"
