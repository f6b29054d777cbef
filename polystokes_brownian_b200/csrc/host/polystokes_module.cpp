// polystokes_module.cpp -- the reference's pybind11 module `PolyStokes`
// (src/bindings.cpp:41-119) over the B200 engine's C-ABI.
//
// Same class, method names, argument names, defaults and output files as the
// reference; the run() loop (src/run.cpp:55-175) calls ps_step once per time
// step.  The noise is drawn on the host exactly as the reference draws it -- a
// std::mt19937_64 seeded with `seed` and one std::normal_distribution<double>,
// nm3nc11 slip draws then nm3nc6 RFD draws per step (slip_vel.cpp:11-17,
// drift.cpp:9-15) -- and passed to ps_step, so a seed gives the reference's
// noise sequence.  Differences from the reference (documented there as its
// conventions): errors raise RuntimeError instead of aborting the process, and
// several simulations may live in one process.
//
// Options the reference does not have (set_options, set_lubrication, state
// accessors) keep their defaults unless called: FP64, structured saddle solve,
// rtol 1e-6 (the reference's hard-coded KSP tolerance, init.cpp:64).
#include <pybind11/iostream.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "polystokes_b200.h"

namespace py = pybind11;

namespace {

void check(int rc, const char *what)
{
    if (rc < 0) throw std::runtime_error(std::string(what) + " failed (" + std::to_string(rc) + "): " + ps_last_error());
}

// Periodic box (src/box.cpp:6-84): orthorhombic minimum image and wrap.
class Box {
public:
    void configure(const std::vector<double> &lengths)
    {
        if (lengths.empty()) { on_ = false; return; }
        if (lengths.size() != 3)
            throw std::invalid_argument("Box::configure expects an empty list (no PBC) or exactly 3 lengths [Lx, Ly, Lz]");
        for (int i = 0; i < 3; i++)
            if (!(lengths[i] > 0.0)) throw std::invalid_argument("Box lengths must be positive");
        for (int i = 0; i < 3; i++) { L_[i] = lengths[i]; Li_[i] = 1.0 / lengths[i]; }
        on_ = true;
    }
    bool active() const { return on_; }
    void minimum_image(double &dx, double &dy, double &dz) const
    {
        if (!on_) return;
        dx -= L_[0] * std::nearbyint(dx * Li_[0]);
        dy -= L_[1] * std::nearbyint(dy * Li_[1]);
        dz -= L_[2] * std::nearbyint(dz * Li_[2]);
    }
    void wrap(double &x, double &y, double &z) const { minimum_image(x, y, z); }
    const double *lengths() const { return L_; }

private:
    bool on_ = false;
    double L_[3] = {0, 0, 0}, Li_[3] = {0, 0, 0};
};

class PolyStokes {
public:
    PolyStokes(double dt, int samplerate, double tmax, std::string output_dir, bool mm_HI, bool chain_HI, bool fene,
               bool record_forces, bool tether, bool mono_ev, const std::vector<double> &box, double t,
               unsigned long seed, double restart)
        : dt_(dt), samplerate_(samplerate), tmax_(tmax), out_(std::move(output_dir)), seed_(seed), restart_(restart)
    {
        std::cout << "using bond force fene: " << fene << std::endl;
        box_.configure(box);
        if (box_.active())
            std::cout << "periodic box: [" << box[0] << ", " << box[1] << ", " << box[2] << "]" << std::endl;
        (void)t;   // the reference keeps `t` but starts the clock at `restart` (Stokes.cpp:21)
        nsteps_ = (long)std::floor((tmax - restart) / dt);
        if (nsteps_ < 0) {
            std::cerr << "Warning: restart (" << restart << ") >= tmax (" << tmax << "); no steps to run." << std::endl;
            nsteps_ = 0;
        }
        if (restart != 0.0)
            std::cout << "restart: resuming at t=" << restart << ", running " << nsteps_ << " steps to t=" << tmax
                      << std::endl;
        d_ = ps_desc{};
        d_.dt = dt;
        d_.mm_HI = mm_HI; d_.chain_HI = chain_HI; d_.fene = fene; d_.record_forces = record_forces;
        d_.tether = tether; d_.mono_ev = mono_ev;
        d_.box_on = box_.active();
        for (int i = 0; i < 3; i++) d_.box[i] = box_.active() ? box_.lengths()[i] : 0.0;
        d_.t0 = restart;
        d_.restart = restart != 0.0;
        d_.weaken_trap = -1;
        d_.hs_kpref = 1.0; d_.hs_kmode = 0; d_.lanczos_nc = 64;
        d_.lub_gap = 0.5;
    }
    ~PolyStokes() { if (ctx_) ps_ctx_destroy(ctx_); }

    void particle_info(double kT, double epsilon, int Np, int Nc, int Nm, int Npoly, int Nmono_per_chain, double beta,
                       double kbond, double r0, double Lmax, double tau)
    {
        d_.kT = kT; d_.epsilon = epsilon; d_.Nc = Nc; d_.Nm = Nm; d_.Npoly = Npoly;
        d_.Nmono_per_chain = Nmono_per_chain; d_.beta = beta; d_.kbond = kbond; d_.r0 = r0; d_.Lmax = Lmax;
        d_.tau = tau;
        Np_ = Np;
        std::cout << "kT: " << kT << "\nepsilon: " << epsilon << "\nNp: " << Np << "\nNc: " << Nc << "\nNm: " << Nm
                  << "\nNpoly: " << Npoly << "\nNmono_per_chain: " << Nmono_per_chain << "\nbeta: " << beta
                  << "\nkbond: " << kbond << "\nr0: " << r0 << "\nLmax: " << Lmax << "\ntau: " << tau << std::endl;
        if (Np != Nm + Nc) throw std::runtime_error("particle_info: Np != Nm + Nc");
        have_pinfo_ = true;
    }

    void trap_info(double ktrap, double tstart, double trun, double weaken_trap)
    {
        d_.ktrap = ktrap; d_.tstart = tstart; d_.trun = trun; d_.weaken_trap = weaken_trap;
        if (tstart + trun > tmax_) std::cerr << "Simulation time exceeds maximum time" << std::endl;
    }

    void initial_configuration(py::array_t<double, py::array::c_style | py::array::forcecast> x0, py::object init_q)
    {
        if (!have_pinfo_) throw std::runtime_error("initial_configuration: call particle_info first");
        auto b = x0.request();
        if ((long)b.size != 3L * Np_) throw std::runtime_error("initial_configuration: init_x0 must hold 3*Np values");
        const double *p = static_cast<const double *>(b.ptr);
        x_.assign(p, p + b.size);
        q_.assign(4L * d_.Nc, 0.0);
        for (int c = 0; c < d_.Nc; c++) q_[4 * c] = 1.0;
        if (restart_ == 0.0) std::cout << "Storing initial positions" << std::endl;
        else std::cout << "restart: trap center kept at origin (not re-derived from the drifted colloid)" << std::endl;
        if (!init_q.is_none()) {
            auto qa = init_q.cast<py::array_t<double, py::array::c_style | py::array::forcecast>>();
            auto qb = qa.request();
            if ((long)qb.size != 4L * d_.Nc) {
                std::cerr << "Warning: init_q size (" << qb.size << ") != Nc*4 (" << 4 * d_.Nc
                          << "); falling back to identity quaternions." << std::endl;
            } else {
                const double *qp = static_cast<const double *>(qb.ptr);
                q_.assign(qp, qp + qb.size);
                std::cout << "restart: restoring " << d_.Nc << " quaternion(s) from init_q" << std::endl;
            }
        }
        have_x_ = true;
    }

    void set_warn_neg_eig(bool on) { warn_neg_eig_ = on; }

    void set_options(const std::string &precision, const std::string &solver, double rtol, const std::string &noise,
                     int ab_mode, int aa_mode, int sqrt_kmax, double sqrt_tol, int maxit, bool strict)
    {
        if (maxit < 1) throw std::invalid_argument("maxit must be >= 1");
        if (precision != "fp64" && precision != "mixed") throw std::invalid_argument("precision: fp64 | mixed");
        if (solver != "minres" && solver != "structured") throw std::invalid_argument("solver: minres | structured");
        if (noise != "host" && noise != "device") throw std::invalid_argument("noise: host | device");
        prec_ = precision == "mixed" ? PS_PREC_MIXED : PS_PREC_FP64;
        solver_ = solver == "minres" ? PS_SOLVE_MINRES : PS_SOLVE_STRUCTURED;
        rtol_ = rtol;
        host_noise_ = noise == "host";
        d_.ab_mode = ab_mode; d_.aa_mode = aa_mode;
        sqrt_kmax_ = sqrt_kmax; sqrt_tol_ = sqrt_tol;
        maxit_ = maxit; strict_ = strict;
    }

    void set_lubrication(py::array_t<double, py::array::c_style | py::array::forcecast> table, double gap, bool bonded)
    {
        auto b = table.request();
        if (b.ndim != 2 || b.shape[1] < 11 || b.shape[0] < 2)
            throw std::invalid_argument("lubrication table: rows of (r, 10 resistance functions) as in lubdat/r2babc.dat");
        const double *p = static_cast<const double *>(b.ptr);
        lub_.assign(p, p + b.size);
        lub_rows_ = (int)b.shape[0];
        lub_cols_ = (int)b.shape[1];
        d_.lub_on = 1; d_.lub_gap = gap; d_.lub_bonded = bonded;
    }

    void run()
    {
        py::scoped_ostream_redirect redirect;
        if (!have_pinfo_ || !have_x_) throw std::runtime_error("run: particle_info and initial_configuration first");
        std::cout << "FTS Stokesian Dynamics (unbounded), B200 engine" << std::endl;
        if (const char *e = std::getenv("HS_KPREF")) d_.hs_kpref = std::atof(e);     // pair_interaction.cpp:185
        if (const char *e = std::getenv("HS_KMODE")) d_.hs_kmode = std::atoi(e);     // pair_interaction.cpp:186
        if (const char *e = std::getenv("POLYSTOKES_LANCZOS_NC")) d_.lanczos_nc = std::atoi(e);   // slip_vel.cpp:97
        if (ctx_) { ps_ctx_destroy(ctx_); ctx_ = nullptr; }
        check(ps_ctx_create(&d_, 1, prec_, &ctx_), "ps_ctx_create");
        if (d_.lub_on) check(ps_set_lub_table(ctx_, lub_.data(), lub_rows_, lub_cols_), "ps_set_lub_table");
        check(ps_set_seed(ctx_, seed_), "ps_set_seed");
        check(ps_set_state(ctx_, x_.data(), d_.Nc ? q_.data() : nullptr, nullptr), "ps_set_state");
        check(ps_set_time(ctx_, restart_), "ps_set_time");
        std::cout << "Initialization complete \n\n" << std::endl;

        const long nm3nc11 = 3L * d_.Nm + 11L * d_.Nc, nm3nc6 = 3L * d_.Nm + 6L * d_.Nc;
        std::mt19937_64 rng(seed_);                       // init.cpp:105-110
        std::normal_distribution<double> normal(0.0, 1.0);
        std::vector<double> fb(nm3nc11), W(nm3nc6), fext(nm3nc6), sb(nm3nc6);
        double t = restart_;
        long neg_stages = 0, neg_total = 0;
        for (long i = 0; i < nsteps_; i++) {
            t += dt_;
            ps_step_inputs in{};
            if (d_.kT > 0 && host_noise_) {
                for (auto &v : fb) v = normal(rng);           // sample_slip_vel
                for (auto &v : W) v = normal(rng);            // sample_drift_displacement
                in.fb = fb.data();
                in.wrfd = W.data();
            }
            in.rtol = rtol_;
            in.maxit = maxit_;
            in.sqrt_kmax = sqrt_kmax_;
            in.sqrt_tol = sqrt_tol_;
            in.solver = solver_;
            ps_step_result res{};
            int rc;
            {
                py::gil_scoped_release nogil;
                rc = ps_step(ctx_, &in, &res, nullptr);
            }
            check(rc, "ps_step");
            if (res.reason < 0) {
                // the reference only reports a failed KSPSolve and carries on (vel.cpp:45-51);
                // with strict set the run stops with the solver's reason instead
                std::cout << "Warning: saddle solve did not converge (reason " << res.reason << ") at t=" << t << std::endl;
                if (strict_) {
                    t_ = t;
                    throw std::runtime_error("run: saddle solve did not converge (KSP reason " +
                                             std::to_string(res.reason) + ") at step " + std::to_string(i + 1));
                }
            }
            if (res.lanczos_nneg > 0) {
                neg_stages++;
                neg_total += res.lanczos_nneg;
                if (warn_neg_eig_)
                    std::printf("[schur/lanczos] floored %ld negative projected eigenvalue(s)\n", (long)res.lanczos_nneg);
            }
            if (i == 0 || i % samplerate_ == 0) {
                check(ps_get_state(ctx_, x_.data(), d_.Nc ? q_.data() : nullptr, nullptr), "ps_get_state");
                check(ps_step_outputs(ctx_, nullptr, nullptr, sb.data(), fext.data(), nullptr), "ps_step_outputs");
                std::cout << "Time " << t << std::endl;
                write_configuration(t);
                write_quaternions(t);
                if (d_.record_forces) write_forces(t, fext);
                write_stresslets(t, sb);
            }
        }
        check(ps_get_state(ctx_, x_.data(), d_.Nc ? q_.data() : nullptr, nullptr), "ps_get_state");
        t_ = t;
        std::printf("[schur:stats] Lanczos noise path floored negatives on %ld stage(s), %ld total.\n", neg_stages,
                    neg_total);
        std::fflush(stdout);
    }

    py::array_t<double> positions() const { return py::array_t<double>(x_.size(), x_.data()); }
    py::array_t<double> quaternions() const { return py::array_t<double>(q_.size(), q_.data()); }
    double time() const { return t_; }

private:
    // file name: output_dir + "/<kind>_" + (time as std::ostream prints a double) + "_.txt"
    std::string fname(const char *kind, double t) const
    {
        std::ostringstream oss;
        oss << out_ << "/" << kind << "_" << t << "_.txt";
        return oss.str();
    }
    static void rows(FILE *f, const double *v, long nrow, int ncol)
    {
        for (long i = 0; i < nrow; i++)
            for (int c = 0; c < ncol; c++) std::fprintf(f, c + 1 < ncol ? "%.10f\t" : "%.10f\n", v[ncol * i + c]);
    }
    FILE *open(const char *kind, double t, const char *who) const
    {
        FILE *f = std::fopen(fname(kind, t).c_str(), "w");
        if (!f) std::cerr << "Error: Could not open the file for writing in " << who << "." << std::endl;
        return f;
    }
    // write_configuration.cpp:10-38
    void write_configuration(double t) const
    {
        if (FILE *f = open("config", t, "write_configuration")) { rows(f, x_.data(), Np_, 3); std::fclose(f); }
    }
    // write_configuration.cpp:40-70
    void write_quaternions(double t) const
    {
        if (FILE *f = open("quats", t, "write_quaternion")) { rows(f, q_.data(), d_.Nc, 4); std::fclose(f); }
    }
    // write_configuration.cpp:72-119: forces of all beads, then colloid torques
    void write_forces(double t, const std::vector<double> &fext) const
    {
        if (FILE *f = open("force", t, "write_configuration")) {
            rows(f, fext.data(), Np_, 3);
            rows(f, fext.data() + 3L * Np_, d_.Nc, 3);
            std::fclose(f);
        }
    }
    // write_configuration.cpp:122-166
    void write_stresslets(double t, const std::vector<double> &sb) const
    {
        if (FILE *f = open("brownian_stresslet", t, "write_stresslets")) { rows(f, sb.data(), d_.Nc, 5); std::fclose(f); }
    }

    double dt_;
    int samplerate_;
    double tmax_;
    std::string out_;
    unsigned long seed_;
    double restart_;
    long nsteps_ = 0;
    Box box_;
    ps_desc d_{};
    int Np_ = 0;
    bool have_pinfo_ = false, have_x_ = false, warn_neg_eig_ = true;
    std::vector<double> x_, q_;
    double t_ = 0.0;
    int prec_ = PS_PREC_FP64, solver_ = PS_SOLVE_STRUCTURED;
    double rtol_ = 1e-6;
    bool host_noise_ = true;
    int sqrt_kmax_ = 40;
    double sqrt_tol_ = 1e-6;
    int maxit_ = 10000;
    bool strict_ = false;
    std::vector<double> lub_;
    int lub_rows_ = 0, lub_cols_ = 0;
    ps_ctx *ctx_ = nullptr;
};

}  // namespace

PYBIND11_MODULE(PolyStokes, m)
{
    m.doc() = "Polymer Stokesian Dynamics simulation module (B200 engine)";
    py::class_<PolyStokes>(m, "PolyStokes")
        .def(py::init([](double dt, int samplerate, double tmax, std::string output_dir, bool mm_HI, bool chain_HI,
                         bool fene, bool record_forces, bool tether, bool mono_ev, py::object box, double t,
                         unsigned long seed, double restart) {
                 std::vector<double> bl;
                 if (!box.is_none()) bl = box.cast<std::vector<double>>();
                 return new PolyStokes(dt, samplerate, tmax, output_dir, mm_HI, chain_HI, fene, record_forces, tether,
                                       mono_ev, bl, t, seed, restart);
             }),
             py::arg("dt"), py::arg("samplerate"), py::arg("tmax"), py::arg("output_dir"), py::arg("mm_HI") = true,
             py::arg("chain_HI") = false, py::arg("fene") = true, py::arg("record_forces") = true,
             py::arg("tether") = false, py::arg("mono_ev") = false, py::arg("box") = py::none(), py::arg("t") = 0.0,
             py::arg("seed") = 12345, py::arg("restart") = 0.0)
        .def("initial_configuration", &PolyStokes::initial_configuration, py::arg("init_x0"),
             py::arg("init_q") = py::none(), "Initialize particle positions; on restart pass init_q (Nc x 4 flattened)")
        .def("particle_info", &PolyStokes::particle_info, py::arg("kT"), py::arg("epsilon"), py::arg("Np"),
             py::arg("Nc"), py::arg("Nm"), py::arg("Npoly"), py::arg("Nmono_per_chain"), py::arg("beta"),
             py::arg("kbond"), py::arg("r0"), py::arg("Lmax"), py::arg("tau"), "Set the parameters for the particles")
        .def("trap_info", &PolyStokes::trap_info, py::arg("ktrap"), py::arg("tstart"), py::arg("trun"),
             py::arg("weaken_trap") = -1, "Set the parameters for the traps")
        .def("run", &PolyStokes::run, "Run the simulation")
        .def("set_warn_neg_eig", &PolyStokes::set_warn_neg_eig, py::arg("on") = true,
             "Toggle per-event negative-eigenvalue warning prints (default on)")
        // not in the reference
        .def("set_options", &PolyStokes::set_options, py::arg("precision") = "fp64", py::arg("solver") = "structured",
             py::arg("rtol") = 1e-6, py::arg("noise") = "host", py::arg("ab_mode") = 0, py::arg("aa_mode") = 0,
             py::arg("sqrt_kmax") = 40, py::arg("sqrt_tol") = 1e-6, py::arg("maxit") = 10000,
             py::arg("strict") = false,
             "Engine options: precision fp64|mixed, solver structured|minres, rtol, noise host (the reference's "
             "mt19937_64 stream) | device (Philox), pair scalars (0 reference, 1 RPY), Lanczos noise cap/tolerance, "
             "solver iteration cap, strict (raise RuntimeError when a saddle solve does not converge; the "
             "reference only prints)")
        .def("set_lubrication", &PolyStokes::set_lubrication, py::arg("table"), py::arg("gap") = 0.5,
             py::arg("bonded") = false, "Near-field lubrication from a lubdat/r2babc.dat table")
        .def("positions", &PolyStokes::positions)
        .def("quaternions", &PolyStokes::quaternions)
        .def("time", &PolyStokes::time);

    py::class_<Box>(m, "Box")
        .def(py::init<>())
        .def("configure", &Box::configure, py::arg("lengths"),
             "Configure the box: [] disables PBC, [Lx,Ly,Lz] enables an orthorhombic cell")
        .def("active", &Box::active)
        .def("minimum_image",
             [](const Box &b, double dx, double dy, double dz) {
                 b.minimum_image(dx, dy, dz);
                 return py::make_tuple(dx, dy, dz);
             },
             py::arg("dx"), py::arg("dy"), py::arg("dz"), "Return the minimum-image of a separation vector")
        .def("wrap",
             [](const Box &b, double x, double y, double z) {
                 b.wrap(x, y, z);
                 return py::make_tuple(x, y, z);
             },
             py::arg("x"), py::arg("y"), py::arg("z"),
             "Return a position wrapped into the primary cell centered at the origin");
}
