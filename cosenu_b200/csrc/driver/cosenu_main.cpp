// cosenu_main -- drop-in for COSEnu's driver (src/main.cpp:58-231) running
// the time loop on the GPU through the C ABI.
//
//   cosenu_main --conf job.config [--ff] [--presets presets.hpp]
//               [--fp32] [--device N] [--checkpoint-every N]
//
// Same inputs (job.config, G0.bin / state.bin / state0.bin with --ff) and the
// same outputs (conserved_quantities.dat, survival_probability.dat,
// rho_<t>.dat, time.txt) as the reference binary.  The physics switches that
// the reference fixes at compile time come from a presets.hpp as manage.py
// writes it (default: the checked-in src/presets.hpp: periodic FV with the
// vacuum and collective terms); the "scheme" key of job.config selects FV/FD
// when no presets file names one.
//
// Differences from the reference: failures exit with status 1 (the
// reference exits 0 on a bad config, src/parser.hpp:220-243); N_ITER < 10
// does not divide by zero in the progress print (src/main.cpp:195); the loop
// advances in chunks between analysis/dump events, which is the same
// sequence of RK4 steps.
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

#include "cosenu_nuosc.hpp"

using namespace cosenu;

int main(int argc, char *argv[])
{
    std::string conf, presets_path;
    bool is_ff = false;
    int precision = COSENU_FP64, device = 0, checkpoint_every = 0;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--conf" && i + 1 < argc) conf = argv[++i];
        else if (a == "--ff") is_ff = true;
        else if (a == "--presets" && i + 1 < argc) presets_path = argv[++i];
        else if (a == "--fp32") precision = COSENU_FP32_BULK;
        else if (a == "--device" && i + 1 < argc) device = std::atoi(argv[++i]);
        else if (a == "--checkpoint-every" && i + 1 < argc) checkpoint_every = std::atoi(argv[++i]);
        else if (a == "--id" && i + 1 < argc) ++i;  // accepted and ignored, as in the reference
    }
    if (conf.empty()) {
        std::cout << "[ FAIL ]...The configuration should be passed on runtime." << std::endl
                  << "Use --conf to specify them." << std::endl
                  << "General format:\n\t$./cosenu_main --conf <Configuration file name> [--ff]\n";
        return 1;
    }
    if (is_ff) std::cout << "Initializing from file.\n";

    std::string perr;
    Presets pr = presets_path.empty() ? Presets::reference_default()
                                      : Presets::parse(presets_path, &perr);
    if (!perr.empty()) {
        std::cout << "[ FAIL ]..." << perr << std::endl;
        return 1;
    }
    JobConfig pars = JobConfig::parse(conf, pr.flags & COSENU_VAC, pr.flags & COSENU_COLL);
    for (const auto &k : pars.unknown_keys) std::cout << "Redundant or unknown key: " << k << std::endl;
    if (!pars.error.empty()) {
        std::cout << pars.error << std::endl << "Exiting." << std::endl;
        return 1;
    }
    if (!pr.scheme_set || presets_path.empty()) {
        if (pars.SCHEME == "FD" || pars.SCHEME == "fd") {
            pr.scheme = COSENU_FD;
            pr.fd_advec = COSENU_FD_CENTER;  // manage.py:168-171 pairs FD with these two
            pr.ko_order = 3;
        } else {
            pr.scheme = COSENU_FV;
        }
    }

    try {
        NuOscGPU state(pars, pr, precision, device);
        const int N_ITER = pars.N_ITER;
        std::cout << "##################################################\n"
                  << "SCHEME: " << pars.SCHEME << "  (Nvz, Nz): (" << pars.nvz << ", " << pars.nz
                  << ")  gz: " << pars.gz << "  CFL: " << pars.CFL << "\n"
                  << "NUMBER OFITERATIONS: " << N_ITER << std::endl;
        int t0;
        if (!is_ff) {
            state.initialize(pars.perturbation_size);
            state.write_state0();
            t0 = 1;
        } else {
            if (!state.read_G0()) {
                std::cout << "G0.bin does not exist. Exiting.\n";
                return 1;
            }
            t0 = state.read_state();
            if (t0 < 0) {
                std::cout << "state0.bin did not open. Exiting.\n";
                return 1;
            }
            if (!state.read_state0()) {
                std::cout << "state0.bin does not exist. Exiting.\n";
                return 1;
            }
        }
        std::cout << "Starting time = " << t0 << "\n";
        if (!is_ff) {
            cosenu_diag d = state.diagnostics();
            state.analyse(0, d);
            state.surv_prob(0, d);
            state.dump_rho(0);
        }

        auto start = std::chrono::steady_clock::now();
        const int progress = std::max(1, N_ITER / 10);
        auto next_multiple = [](int t, int m) { return m > 0 ? ((t + m - 1) / m) * m : 1 << 30; };
        int t_iter = t0;
        while (t_iter < N_ITER) {
            // the next iteration at which the reference would do host work
            int ev = N_ITER - 1;
            ev = std::min(ev, next_multiple(t_iter, pars.ANAL_EVERY));
            ev = std::min(ev, next_multiple(t_iter, pars.dump_interval));
            ev = std::min(ev, next_multiple(t_iter, progress));
            if (checkpoint_every > 0) ev = std::min(ev, next_multiple(t_iter, checkpoint_every));
            state.advance(ev - t_iter + 1);
            t_iter = ev;
            if (t_iter % pars.ANAL_EVERY == 0) {
                cosenu_diag d = state.diagnostics();
                state.analyse(t_iter, d);
                state.surv_prob(t_iter, d);
            }
            state.write_output(t_iter, t_iter % pars.dump_interval == 0,
                               checkpoint_every > 0 && t_iter % checkpoint_every == 0);
            if (t_iter % progress == 0)
                std::cout << " " << std::setprecision(4)
                          << (int)(t_iter * 100.0 / (N_ITER - 1)) << " %" << std::endl;
            ++t_iter;
        }
        cosenu_synchronize(state.ctx());
        state.finish_output();
        auto end = std::chrono::steady_clock::now();
        std::chrono::duration<double> el = end - start;
        std::cout << " 100 %" << std::endl << std::endl << "SIMULATION COMPLETED" << std::endl;
        std::ofstream xtf("time.txt", std::ofstream::out | std::ofstream::trunc);
        xtf << el.count() << std::endl;
        std::cout << "elapsed time: " << el.count() << "s\n";
    } catch (const Error &e) {
        std::cout << "[ FAIL ]..." << e.what() << std::endl;
        return 1;
    }
    return 0;
}
