// cosenu_nuosc.hpp -- host-side mirror of COSEnu's NuOsc / Params over the
// C ABI of cosenu_b200.h (header-only, C++17).
//
//  * JobConfig  : the job.config parser of src/parser.hpp:46-256 (same keys,
//                 same required set, same dump_interval rule); it reports a
//                 missing key through an error string instead of exit(0).
//  * Presets    : reads the compile-time switches manage.py writes into
//                 src/presets.hpp (manage.py:160-186) so one binary serves
//                 every variant.
//  * NuOscGPU   : NuOsc (src/nuosc.hpp:7-191) with the state on the GPU:
//                 initialize / read_G0 / read_state / read_state0 /
//                 write_state / write_state0 / step_rk4 / analyse /
//                 surv_prob / dump_rho with the reference's file formats
//                 (src/snaps.hpp, src/analysis.hpp).  rho_<t>.dat and the
//                 state.bin checkpoint are written from a device snapshot by
//                 a host thread while the GPU keeps stepping.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "cosenu_b200.h"
#include "cosenu_format.hpp"

namespace cosenu {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

// ---------------------------------------------------------------------------
struct JobConfig {
    std::string SCHEME;
    int N_ITER = 0, ANAL_EVERY = 0, nz = 0, nvz = 0, gz = 0;
    double z0 = 0.0, z1 = 0.0, v0 = 0.0, v1 = 0.0, CFL = 0.0, pmo = 0.0, omega = 0.0,
           theta = 0.0, mu = 1.0, perturbation_size = 0.0;
    int n_dump = 0, dump_interval = 0;
    std::vector<std::string> unknown_keys;
    std::string error;  // empty when the file was complete

    // src/parser.hpp:99-256; `need_vac` / `need_coll` mirror the VAC_OSC_ON /
    // COLL_OSC_ON checks at :235-243.
    static JobConfig parse(const std::string &path, bool need_vac, bool need_coll)
    {
        JobConfig c;
        std::ifstream f(path.c_str());
        if (!f) {
            c.error = "[ FAIL ]...Unable to open " + path;
            return c;
        }
        bool h[32] = {false};
        enum { SCH, NZ, NVZ, Z0, Z1, V0, V1, CFLK, GZ, NIT, ANA, PMO, OMG, THE, MU };
        std::string line, key, value;
        while (std::getline(f, line)) {
            if (line.empty()) continue;
            size_t pos = line.find_first_of(':');
            std::string left = line.substr(0, pos);
            std::string right = pos == std::string::npos ? std::string() : line.substr(pos + 1);
            if (!left.empty()) {
                key = left.substr(0, left.find_first_of(' '));
                size_t b = right.find_first_not_of(' ');
                value = b == std::string::npos ? std::string() : right.substr(b);
            }
            std::stringstream sv(value);
            if (key == "scheme") { sv >> c.SCHEME; h[SCH] = true; }
            else if (key == "nz") { sv >> c.nz; h[NZ] = true; }
            else if (key == "nvz") { sv >> c.nvz; h[NVZ] = true; }
            else if (key == "CFL") { sv >> c.CFL; h[CFLK] = true; }
            else if (key == "gz") { sv >> c.gz; h[GZ] = true; }
            else if (key == "z0") { sv >> c.z0; h[Z0] = true; }
            else if (key == "z1") { sv >> c.z1; h[Z1] = true; }
            else if (key == "v0") { sv >> c.v0; h[V0] = true; }
            else if (key == "v1") { sv >> c.v1; h[V1] = true; }
            else if (key == "perturbation_size") { sv >> c.perturbation_size; }
            else if (key == "N_ITER") { sv >> c.N_ITER; h[NIT] = true; }
            else if (key == "ANAL_EVERY") { sv >> c.ANAL_EVERY; h[ANA] = true; }
            else if (key == "pmo") { sv >> c.pmo; h[PMO] = true; }
            else if (key == "omega") { sv >> c.omega; h[OMG] = true; }
            else if (key == "theta") { sv >> c.theta; h[THE] = true; }
            else if (key == "mu") { sv >> c.mu; h[MU] = true; }
            else if (key == "n_dump_rho") { sv >> c.n_dump; }
            else c.unknown_keys.push_back(key);
        }
        bool ok = h[SCH] && h[NZ] && h[NVZ] && h[Z0] && h[Z1] && h[V0] && h[V1] && h[CFLK] &&
                  h[GZ] && h[NIT] && h[ANA];
        if (need_vac) ok = ok && h[PMO] && h[OMG] && h[THE];
        if (need_coll) ok = ok && h[MU];
        if (!ok) c.error = "[ FAIL ]...Incomplete config file";
        if (c.n_dump > 0) {
            c.dump_interval = (int)(c.N_ITER / c.n_dump);
            if (c.dump_interval < 1) c.dump_interval = 1;
        } else {
            c.dump_interval = c.N_ITER + 1;
        }
        return c;
    }
};

// ---------------------------------------------------------------------------
struct Presets {
    int scheme = COSENU_FV, bc = COSENU_PERIODIC, fd_advec = COSENU_FD_LOPSIDED, ko_order = 5;
    unsigned flags = 0;
    bool scheme_set = false;

    // The checked-in default, src/presets.hpp:1-9.
    static Presets reference_default()
    {
        Presets p;
        p.scheme = COSENU_FV;
        p.bc = COSENU_PERIODIC;
        p.flags = COSENU_VAC | COSENU_COLL;
        p.scheme_set = true;
        return p;
    }

    // Reads the #define lines of a presets.hpp as manage.py writes it.  FD
    // without ADVEC_CENTER_FD / ADVEC_UPWIND selects the lopsided stencil and
    // without KO_ORD_3 the 5th-order dissipation, as in src/rhs_fd.hpp.
    static Presets parse(const std::string &path, std::string *err)
    {
        Presets p;
        std::ifstream f(path.c_str());
        if (!f) {
            if (err) *err = "cannot open presets file " + path;
            return reference_default();
        }
        std::string line;
        bool fd = false, fv = false, center = false, upwind = false, ko3 = false, open = false;
        while (std::getline(f, line)) {
            std::stringstream ss(line);
            std::string d, name;
            ss >> d >> name;
            if (d != "#define") continue;
            if (name == "FD") fd = true;
            else if (name == "FV") fv = true;
            else if (name == "OPEN_BC") open = true;
            else if (name == "ADVEC_CENTER_FD") center = true;
            else if (name == "ADVEC_UPWIND") upwind = true;
            else if (name == "KO_ORD_3") ko3 = true;
            else if (name == "VAC_OSC_ON") p.flags |= COSENU_VAC;
            else if (name == "MAT_OSC_ON") p.flags |= COSENU_MAT;
            else if (name == "COLL_OSC_ON") p.flags |= COSENU_COLL;
            else if (name == "ADVEC_OFF") p.flags |= COSENU_ADVEC_OFF;
        }
        p.scheme = fd ? COSENU_FD : COSENU_FV;
        p.scheme_set = fd || fv;
        p.bc = open ? COSENU_OPEN : COSENU_PERIODIC;
        p.fd_advec = center ? COSENU_FD_CENTER : (upwind ? COSENU_FD_UPWIND : COSENU_FD_LOPSIDED);
        p.ko_order = ko3 ? 3 : 5;
        return p;
    }
};

// ---------------------------------------------------------------------------
class NuOscGPU {
  public:
    static constexpr int NC = COSENU_NCOMP;
    int nz, nvz, gz, size;
    double dz, dv, dt, phy_time = 0.0;
    std::vector<double> Z, vz;
    // host copies in the reference layout (filled on demand)
    std::vector<double> v_stat, v_stat0, G, bG;

    NuOscGPU(const JobConfig &c, const Presets &pr, int precision = COSENU_FP64, int device = 0)
    {
        cosenu_params p;
        cosenu_params_default(&p);
        p.nz = c.nz;
        p.nvz = c.nvz;
        p.gz = c.gz;
        p.z0 = c.z0;
        p.z1 = c.z1;
        p.v0 = c.v0;
        p.v1 = c.v1;
        p.cfl = c.CFL;
        p.pmo = c.pmo;
        p.omega = c.omega;
        p.theta_deg = c.theta;
        p.mu = c.mu;
        p.scheme = pr.scheme;
        p.bc = pr.bc;
        p.flags = pr.flags;
        p.fd_advec = pr.fd_advec;
        p.ko_order = pr.ko_order;
        p.precision = precision;
        p.device = device;
        int rc = cosenu_create(&p, &ctx_);
        if (rc != COSENU_OK) throw Error(rc, cosenu_last_error(nullptr));
        nz = c.nz;
        nvz = c.nvz;
        gz = c.gz;
        size = (nz + 2 * gz) * nvz;
        double g[5];
        cosenu_grid(ctx_, g);
        dz = g[0];
        dv = g[1];
        dt = g[2];
        Z.resize(nz);
        vz.resize(nvz);
        for (int j = 0; j < nz; ++j) Z[j] = c.z0 + (j + 0.5) * dz;   // src/nuosc.hpp:83-86
        for (int i = 0; i < nvz; ++i) vz[i] = c.v0 + (i + 0.5) * dv;  // src/nuosc.hpp:88-92
        v_stat.assign((size_t)NC * size, 0.0);
        v_stat0.assign((size_t)NC * size, 0.0);
        G.assign(size, 0.0);
        bG.assign(size, 0.0);
    }
    ~NuOscGPU()
    {
        if (writer_.joinable()) writer_.join();
        cosenu_destroy(ctx_);
    }
    NuOscGPU(const NuOscGPU &) = delete;
    NuOscGPU &operator=(const NuOscGPU &) = delete;

    cosenu_ctx *ctx() { return ctx_; }
    int idx(int i, int j) const { return i * (nz + 2 * gz) + (j + gz); }

    void set_vac_pars(double pmo, double omega, double theta_deg)
    {
        check(cosenu_set_vac_pars(ctx_, pmo, omega, theta_deg));
    }
    void set_collective_pars(double mu) { check(cosenu_set_collective_pars(ctx_, mu)); }

    // NuOsc::initialize (src/initialize.hpp:6-47) on the device; also writes
    // G0.bin like the reference.
    void initialize(double perturbation_size)
    {
        check(cosenu_init_reference(ctx_, perturbation_size));
        download_state();
        fetch_profile_from_state_init(perturbation_size);
        std::ofstream g("G0.bin", std::ios::out | std::ios::binary);
        for (int i = 0; i < nvz; ++i)
            for (int j = 0; j < nz; ++j) {
                g.write((const char *)&G[idx(i, j)], sizeof(double));
                g.write((const char *)&bG[idx(i, j)], sizeof(double));
            }
        std::cout << "Simulation state initialized." << std::endl;
    }

    void step_rk4() { advance(1); }
    void advance(int n)
    {
        check(cosenu_step(ctx_, n));
        phy_time += n * dt;
    }

    // -- binary files (src/snaps.hpp) ---------------------------------------
    // write_state: int32 iteration then 8 interleaved doubles per cell,
    // written to state<t>.bin and renamed to state.bin (:6-39).  `t` is the
    // iteration just completed; the header holds t + 1, the iteration a run
    // resumed from the file (read_state) starts at -- the meaning state0.bin
    // has with its implied t = 1 -- so a resumed run repeats no step.
    void write_state(unsigned int t) { write_output(t, false, true); }
    void write_state0()
    {
        std::ofstream f("state0.bin", std::ios::out | std::ios::binary);
        if (!f) throw Error(COSENU_ERR_ARG, "cannot open state0.bin");
        write_cells(f, v_stat0);
    }
    // read_state: state.bin if present (returns its iteration), else
    // state0.bin with t = 1 (:75-124).  Returns -1 when neither opens.
    int read_state()
    {
        int t = 1;
        std::ifstream f("state.bin", std::ios::in | std::ios::binary);
        if (f) {
            f.read((char *)&t, sizeof(int));
            std::cout << "Loading from state.bin. \n";
        } else {
            std::cout << "Unable to find state.bin\nLoading from state0.bin. \n";
            f.open("state0.bin", std::ios::in | std::ios::binary);
            if (!f) return -1;
            t = 1;
        }
        if (!read_cells(f, v_stat)) return -1;
        upload_state();
        return t;
    }
    bool read_state0()
    {
        std::ifstream f("state0.bin", std::ios::in | std::ios::binary);
        if (!f || !read_cells(f, v_stat0)) return false;
        const double *c[NC];
        for (int k = 0; k < NC; ++k) c[k] = v_stat0.data() + (size_t)k * size;
        check(cosenu_set_state0(ctx_, c, gz));
        return true;
    }
    bool read_G0()
    {
        std::ifstream f("G0.bin", std::ios::in | std::ios::binary);
        if (!f) return false;
        for (int i = 0; i < nvz; ++i)
            for (int j = 0; j < nz; ++j) {
                f.read((char *)&G[idx(i, j)], sizeof(double));
                f.read((char *)&bG[idx(i, j)], sizeof(double));
            }
        if (!f) return false;
        check(cosenu_set_profile(ctx_, G.data(), bG.data(), gz));
        return true;
    }

    // -- analysis files (src/analysis.hpp) -----------------------------------
    cosenu_diag diagnostics()
    {
        cosenu_diag d;
        check(cosenu_analyse(ctx_, &d));
        return d;
    }
    // NuOsc::analyse -> dcon (:71-130): conserved_quantities.dat
    void analyse(unsigned int t, const cosenu_diag &d)
    {
        std::ofstream o;
        const char *fn = "conserved_quantities.dat";
        o.open(fn, t == 0 ? std::ofstream::out | std::ofstream::trunc
                          : std::ofstream::out | std::ofstream::app);
        if (!o) {
            std::cout << "Unable to open " << fn << std::endl;
            return;
        }
        if (t == 0) o << "# [time, dP_max(t), <dP>(t), <dbP(t), <dP>(t), |M0|]\n";
        o << t << "\t" << std::fixed << std::setprecision(20) << d.dP_max << "\t" << d.avdP
          << "\t" << d.avbdP << "\t" << d.M0 << std::endl;
    }
    // NuOsc::surv_prob (:134-185): survival_probability.dat
    void surv_prob(unsigned int t, const cosenu_diag &d)
    {
        std::ofstream o;
        const char *fn = "survival_probability.dat";
        if (t == 0) {
            o.open(fn, std::ofstream::out | std::ofstream::trunc);
            if (!o) {
                std::cout << "Unable to open " << fn << std::endl;
                return;
            }
            o << "# [time, <Pee>, <Pbee>]" << std::endl;
        } else {
            o.open(fn, std::ofstream::out | std::ofstream::app);
        }
        if (!o) {
            std::cout << "Unable to open " << fn << std::endl;
            return;
        }
        o << t << "\t" << std::scientific << d.Pee << "\t" << d.Pbee << std::endl;
    }
    // NuOsc::dump_rho (src/snaps.hpp:187-218): rho_<t>.dat, z outer, v inner.
    void dump_rho(unsigned int t) { write_output(t, true, false); }

    // rho_<t>.dat (rho) and/or the state.bin checkpoint (state) of the current
    // state, from one snapshot: the device copies the state aside and the file
    // is formatted and written by a host thread while stepping continues.
    // Waits for the previous output first (its host buffer is reused).
    void write_output(unsigned int t, bool rho, bool state)
    {
        if (!rho && !state) return;
        finish_output();
        check(cosenu_snapshot(ctx_, nullptr));
        writer_ = std::thread([this, t, rho, state] {
            const double *d = nullptr;
            if (cosenu_snapshot_wait(ctx_, &d) != COSENU_OK) {
                writer_err_ = "snapshot copy to the host failed";
                return;
            }
            const double *comp[NC];
            for (int k = 0; k < NC; ++k) comp[k] = d + (size_t)k * nvz * nz;
            if (rho) {
                const std::string fn = "rho_" + std::to_string(t) + ".dat";
                if (!format_rho(fn, nz, nvz, Z.data(), vz.data(), comp, nz))
                    writer_msg_ += "Unable to open " + fn + "\n";
            }
            if (state && !write_state_file(t + 1, comp))
                writer_err_ = "cannot write state" + std::to_string(t + 1) + ".bin";
        });
    }
    // Waits for the output thread; throws if it failed to write a checkpoint.
    void finish_output()
    {
        if (writer_.joinable()) writer_.join();
        if (!writer_msg_.empty()) std::cout << writer_msg_;
        writer_msg_.clear();
        if (!writer_err_.empty()) {
            std::string e;
            e.swap(writer_err_);
            throw Error(COSENU_ERR_ARG, e);
        }
    }

    void download_state()
    {
        double *c[NC];
        for (int k = 0; k < NC; ++k) c[k] = v_stat.data() + (size_t)k * size;
        check(cosenu_download(ctx_, c, gz));
    }
    void upload_state()
    {
        const double *c[NC];
        for (int k = 0; k < NC; ++k) c[k] = v_stat.data() + (size_t)k * size;
        check(cosenu_upload(ctx_, c, gz));
    }

  private:
    cosenu_ctx *ctx_ = nullptr;

    void check(int rc)
    {
        if (rc != COSENU_OK) throw Error(rc, cosenu_last_error(ctx_));
    }
    std::thread writer_;
    std::string writer_err_, writer_msg_;

    // state.bin body (src/snaps.hpp:6-39): int32 iteration, then the 8
    // components interleaved per cell, v-major; written to state<t>.bin and
    // renamed into place.
    bool write_state_file(unsigned int t, const double *const comp[NC])
    {
        const std::string tmp = "state" + std::to_string(t) + ".bin";
        FILE *f = std::fopen(tmp.c_str(), "wb");
        if (!f) return false;
        bool ok = std::fwrite(&t, sizeof(int), 1, f) == 1;
        std::vector<double> row((size_t)nz * NC);
        for (int i = 0; i < nvz && ok; ++i) {
            for (int j = 0; j < nz; ++j)
                for (int k = 0; k < NC; ++k) row[(size_t)j * NC + k] = comp[k][(size_t)i * nz + j];
            ok = std::fwrite(row.data(), sizeof(double), row.size(), f) == row.size();
        }
        ok = (std::fclose(f) == 0) && ok;
        return ok && std::rename(tmp.c_str(), "state.bin") == 0;
    }
    void write_cells(std::ofstream &f, const std::vector<double> &s)
    {
        for (int i = 0; i < nvz; ++i)
            for (int j = 0; j < nz; ++j)
                for (int k = 0; k < NC; ++k)
                    f.write((const char *)&s[(size_t)k * size + idx(i, j)], sizeof(double));
    }
    bool read_cells(std::ifstream &f, std::vector<double> &s)
    {
        for (int i = 0; i < nvz; ++i)
            for (int j = 0; j < nz; ++j)
                for (int k = 0; k < NC; ++k)
                    f.read((char *)&s[(size_t)k * size + idx(i, j)], sizeof(double));
        return (bool)f;
    }
    // The profile the device computed for initialize(): recomputed on the host
    // with the same formula for G0.bin (src/initialize.hpp:26-27,42-43).
    void fetch_profile_from_state_init(double)
    {
        for (int i = 0; i < nvz; ++i) {
            double g = gauss_profile(vz[i], 1.0, 0.6), bg = 0.90 * gauss_profile(vz[i], 1.0, 0.6);
            for (int j = 0; j < nz; ++j) {
                G[idx(i, j)] = g;
                bG[idx(i, j)] = bg;
            }
        }
        v_stat0 = v_stat;
    }
    static double gauss_profile(double v, double v0, double sigma)
    {
        double e = (v - v0) * (v - v0) / (2.0 * sigma * sigma);
        double N = sigma * std::sqrt(M_PI / 2.0) *
                   (std::erf((1.0 + v0) / sigma / std::sqrt(2.0)) +
                    std::erf((1.0 - v0) / sigma / std::sqrt(2.0)));
        return std::exp(-e) / N;
    }
};

}  // namespace cosenu
