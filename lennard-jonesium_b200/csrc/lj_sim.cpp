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
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lj_gpu.h"

namespace {

// fmt's "{}" for a double: the shortest digits that round-trip, fixed notation
// when the decimal exponent is in [-4, 16), scientific ("1e-05") otherwise, no
// trailing ".0" for whole numbers.
std::string fmt_double(double v) {
    if (std::isnan(v)) return "nan";
    if (std::isinf(v)) return v < 0 ? "-inf" : "inf";
    if (v == 0) return std::signbit(v) ? "-0" : "0";
    char buf[64];
    auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::scientific);
    std::string sci(buf, r.ptr);
    size_t epos = sci.find('e');
    std::string mant = sci.substr(0, epos);
    int exp = std::stoi(sci.substr(epos + 1));
    bool neg = mant[0] == '-';
    if (neg) mant = mant.substr(1);
    std::string digits;
    for (char ch : mant)
        if (ch != '.') digits += ch;
    std::string out;
    if (exp >= -4 && exp < 16) {
        if (exp < 0) {
            out = "0." + std::string(-exp - 1, '0') + digits;
        } else if ((int)digits.size() <= exp + 1) {
            out = digits + std::string(exp + 1 - digits.size(), '0');
        } else {
            out = digits.substr(0, exp + 1) + "." + digits.substr(exp + 1);
        }
    } else {
        out = digits.substr(0, 1);
        if (digits.size() > 1) out += "." + digits.substr(1);
        char eb[16];
        std::snprintf(eb, sizeof eb, "e%c%02d", exp < 0 ? '-' : '+', std::abs(exp));
        out += eb;
    }
    return neg ? "-" + out : out;
}

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
    void thermo_row(int step, const lj_thermo& r) {
        std::string s = std::to_string(step) + "," + fmt_double(r.time) + "," + fmt_double(r.kinetic_energy) + "," +
                        fmt_double(r.potential_energy) + "," + fmt_double(r.total_energy) + "," +
                        fmt_double(r.virial) + "," + fmt_double(r.temperature) + "," +
                        fmt_double(r.mean_square_displacement) + "\n";
        std::fputs(s.c_str(), thermo);
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

extern "C" {

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
    if ((rc = lj_gpu_upload_state(ctx, x.data(), v.data(), nullptr, nullptr, 4, 0.0, 0.0, 0.0))) {
        lj_gpu_destroy(ctx);
        return rc;
    }

    Sinks out;
    out.echo = echo;
    out.events = std::fopen(cfg->event_log, "w");
    out.thermo = std::fopen(cfg->thermodynamic_log, "w");
    out.obs = std::fopen(cfg->observation_log, "w");
    out.snap = std::fopen(cfg->snapshot_log, "w");
    if (!out.events || !out.thermo || !out.obs || !out.snap) {
        out.close();
        lj_gpu_destroy(ctx);
        return LJ_ERR_ARG;
    }
    std::fputs("TimeStep,Time,KineticEnergy,PotentialEnergy,TotalEnergy,Virial,Temperature,MeanSquareDisplacement\n",
               out.thermo);
    std::fputs("TimeStep,Temperature,Density,TotalEnergy,Pressure,SpecificHeat,DiffusionCoefficient\n", out.obs);
    std::fputs("TimeStep,ParticleID,Position,Position,Position,Velocity,Velocity,Velocity,Force,Force,Force\n",
               out.snap);
    std::fputs("TimeStep,ParticleID,X,Y,Z,X,Y,Z,X,Y,Z\n", out.snap);

    int time_step = 0;
    int outcome = 0, nobs = 0;
    bool aborted = false;
    std::vector<lj_thermo> recs;
    const char* names[2] = {cfg->eq_name ? cfg->eq_name : "Equilibration Phase",
                            cfg->ob_name ? cfg->ob_name : "Observation Phase"};
    for (int phase = 0; phase < 2 && !aborted && rc == LJ_OK; ++phase) {
        bool eq = phase == 0;
        out.event(time_step, std::string("Phase started: ") + names[phase]);
        int start = time_step, last_check = time_step, last_adjust = time_step, last_obs = time_step;
        int count = 0;
        Window Tw(eq ? cfg->eq_sample_size : cfg->ob_sample_size);
        Window Ew(cfg->ob_sample_size), Ww(cfg->ob_sample_size), tw(cfg->ob_sample_size), mw(cfg->ob_sample_size);
        bool done = false;
        while (!done) {
            // steps until the next step at which this phase can act
            int next = eq ? std::min({last_check + cfg->eq_adjustment_interval, last_adjust + cfg->eq_steady_state_time,
                                      start + cfg->eq_timeout})
                          : last_obs + cfg->ob_observation_interval;
            int K = std::max(1, next - time_step);
            recs.resize((size_t)K);
            if ((rc = lj_gpu_step(ctx, K, recs.data()))) break;
            for (int k = 0; k < K && !done; ++k) {
                const lj_thermo& r = recs[(size_t)k];
                out.thermo_row(time_step, r);  // logged before the increment (simulation_controller.cpp:65-67)
                time_step += 1;
                if (eq) {
                    Tw.push(r.temperature);
                    if (time_step - last_check >= cfg->eq_adjustment_interval) {
                        last_check = time_step;
                        double Tm = Tw.mean();
                        if (relative_error(Tm, cfg->temperature) >= cfg->eq_tolerance) {
                            last_adjust = time_step;
                            if ((rc = lj_gpu_set_temperature(ctx, cfg->temperature, nullptr))) {
                                done = true;
                                break;
                            }
                            out.event(time_step, "Temperature measured at: " + fmt_g4(Tm) +
                                                     ", adjusted to: " + fmt_g4(cfg->temperature));
                        }
                    }
                    if (time_step - last_adjust >= cfg->eq_steady_state_time) {
                        out.event(time_step, std::string("Phase complete: ") + names[phase]);
                        done = true;
                    } else if (time_step - start >= cfg->eq_timeout) {
                        out.event(time_step, "Simulation aborted: Could not equilibrate");
                        done = aborted = true;
                        outcome = 1;
                    }
                } else {
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
                            done = aborted = true;
                            outcome = 2;
                            continue;
                        }
                        ++count;
                        ++nobs;
                        out.obs_row(time_step, o);
                        out.event(time_step, "Observation recorded");
                    }
                    if (count >= cfg->ob_observation_count) {
                        out.event(time_step, std::string("Phase complete: ") + names[phase]);
                        done = true;
                    }
                }
            }
        }
    }
    // snapshot of the final (or aborted) state (simulation_controller.cpp:100-108, :128-134)
    if (rc == LJ_OK) {
        std::vector<double> F(4 * (size_t)N);
        if ((rc = lj_gpu_download_state(ctx, x.data(), v.data(), nullptr, F.data(), 4, nullptr, nullptr, nullptr)) ==
            LJ_OK) {
            std::string step = std::to_string(time_step) + ",";
            std::string line;
            for (int i = 0; i < N; ++i) {
                line = step + std::to_string(i);
                for (const double* a : {x.data(), v.data(), F.data()})
                    for (int k = 0; k < 3; ++k) line += "," + fmt_double(a[4 * (size_t)i + k]);
                line += "\n";
                std::fputs(line.c_str(), out.snap);
            }
        }
    }
    out.close();
    lj_gpu_destroy(ctx);
    if (result) {
        result->time_steps = time_step;
        result->outcome = outcome;
        result->observations = nobs;
        result->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    return rc;
}

}  // extern "C"
