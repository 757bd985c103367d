// Prints, as one JSON object, what include/cosenu_nuosc.hpp's JobConfig and
// Presets parsers read from a job.config and a presets.hpp.
// usage: parse_main <job.config> <presets.hpp> <need_vac 0|1> <need_coll 0|1>
#include <cstdio>
#include <cstdlib>

#include "cosenu_nuosc.hpp"

int main(int argc, char **argv)
{
    if (argc != 5) return 2;
    const cosenu::JobConfig c =
        cosenu::JobConfig::parse(argv[1], std::atoi(argv[3]) != 0, std::atoi(argv[4]) != 0);
    std::string err;
    const cosenu::Presets p = cosenu::Presets::parse(argv[2], &err);
    std::printf("{\"scheme\": \"%s\", \"N_ITER\": %d, \"ANAL_EVERY\": %d, \"nz\": %d, "
                "\"nvz\": %d, \"gz\": %d, \"z0\": %.17g, \"z1\": %.17g, \"v0\": %.17g, "
                "\"v1\": %.17g, \"CFL\": %.17g, \"pmo\": %.17g, \"omega\": %.17g, "
                "\"theta\": %.17g, \"mu\": %.17g, \"perturbation_size\": %.17g, "
                "\"n_dump\": %d, \"dump_interval\": %d, \"error\": \"%s\", "
                "\"p_scheme\": %d, \"p_bc\": %d, \"p_fd_advec\": %d, \"p_ko_order\": %d, "
                "\"p_flags\": %u, \"p_error\": \"%s\"}\n",
                c.SCHEME.c_str(), c.N_ITER, c.ANAL_EVERY, c.nz, c.nvz, c.gz, c.z0, c.z1, c.v0,
                c.v1, c.CFL, c.pmo, c.omega, c.theta, c.mu, c.perturbation_size, c.n_dump,
                c.dump_interval, c.error.c_str(), p.scheme, p.bc, p.fd_advec, p.ko_order,
                p.flags, err.c_str());
    return 0;
}
