// Command-line driver with the reference's run sequence (src/main.cpp:10-104), written against the C
// ABI in include/ddamg.h only: it reads the same seven answers from standard input (ranks_x, ranks_t,
// levels, m0, configuration file, right-hand-side file, parameters file), then runs Methods::CG,
// FGMRES with the V-cycle and FGMRES with the K-cycle (src/methods.cpp:42-190) and checks both
// multigrid solutions the way Methods::check_solution does, writing the two metadata files after the
// checks as the reference does (writeMetadata).  The lattice size, a compile-time
// constant of the reference (include/config.h), is the pair of command-line arguments.  There is one
// GPU and no MPI: ranks_x and ranks_t are read and reported, not used.
//
//   ddamg_main Nx Nt [x_out.bin] < answers.txt
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "ddamg.h"

static void die(const char* what, ddamg_status st) {
    std::cerr << what << " failed (" << st << "): " << ddamg_last_error() << std::endl;
    std::exit(1);
}
#define CHECK(call)                              \
    do {                                         \
        ddamg_status st__ = (call);              \
        if (st__ != DDAMG_OK) die(#call, st__);  \
    } while (0)

static double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Methods::check_solution (src/methods.cpp:173-190): every component of D x within 1e-6 of b
static void check_solution(ddamg_t* h, const std::vector<double>& x, const std::vector<double>& b, int Nt) {
    std::vector<double> Dx(x.size());
    CHECK(ddamg_apply_dirac(h, 0, x.data(), Dx.data(), 1));
    double rr = 0.0, bb = 0.0;
    for (size_t i = 0; i < x.size() / 2; i++) {
        const double dre = Dx[2 * i] - b[2 * i], dim = Dx[2 * i + 1] - b[2 * i + 1];
        rr += dre * dre + dim * dim;
        bb += b[2 * i] * b[2 * i] + b[2 * i + 1] * b[2 * i + 1];
        if (std::sqrt(dre * dre + dim * dim) > 1e-6) {
            const size_t site = i / 2;
            std::cout << "Solution differs at nx" << site / Nt + 1 << " nt " << site % Nt + 1 << " mu " << i % 2
                      << std::endl;
        }
    }
    std::printf("Solution verified (||D x - b|| / ||b|| = %.3e)\n", std::sqrt(rr / bb));
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::cerr << "usage: ddamg_main Nx Nt [x_out.bin] < answers (ranks_x ranks_t levels m0 conf rhs params)\n";
        return 2;
    }
    const int Nx = std::atoi(argv[1]), Nt = std::atoi(argv[2]);
    int ranks_x = 1, ranks_t = 1, levels = 2;
    double m0 = 0.0;
    std::string confFile, rhsFile, pFile;
    std::cout << " -----------------------------" << std::endl;
    std::cout << "| DDalpha-AMG Schwinger Model |" << std::endl;
    std::cout << " -----------------------------" << std::endl;
    std::cout << "Nx " << Nx << " Nt " << Nt << std::endl;
    std::cin >> ranks_x >> ranks_t >> levels >> m0 >> confFile >> rhsFile >> pFile;
    if (!std::cin) {
        std::cerr << "expected: ranks_x ranks_t levels m0 conf rhs params on standard input\n";
        return 2;
    }
    std::cout << "ranks_x " << ranks_x << " ranks_t " << ranks_t << " (one GPU: SAP domains map to thread blocks)\n";

    ddamg_params p;
    CHECK(ddamg_params_default(&p));
    p.Nx = Nx;
    p.Nt = Nt;
    p.m0 = m0;
    CHECK(ddamg_parse_params_file(pFile.c_str(), levels, &p));
    const size_t n = 2ul * Nx * Nt;  // complex values of a fine field
    std::vector<double> U(2 * n), b(2 * n), x(2 * n, 0.0), phi(2 * n);
    CHECK(ddamg_read_binary(confFile.c_str(), Nx, Nt, U.data()));
    CHECK(ddamg_read_binary(rhsFile.c_str(), Nx, Nt, b.data()));
    const double tol = 1e-10;

    ddamg_t* h = nullptr;
    CHECK(ddamg_create(&p, &h));
    CHECK(ddamg_load_gauge(h, U.data()));

    // Methods::CG: CG::max_iter = 20000, CG on D^dagger D x = D^dagger b
    std::cout << "--------Inverting the normal equations with CG----------" << std::endl;
    ddamg_solve_info info;
    CHECK(ddamg_apply_dirac(h, 1, b.data(), phi.data(), 1));
    double t0 = now();
    ddamg_status st = ddamg_cg_normal(h, phi.data(), x.data(), 20000, tol, &info);
    if (st != DDAMG_OK && st != DDAMG_NOT_CONVERGED) die("ddamg_cg_normal", st);
    std::printf("CG for D^+D %s in %d iterations\n", info.converged ? "converged" : "did not converge",
                info.iterations);
    std::printf("time elapsed CG: %.4fs.\n\n", now() - t0);

    // the run's iteration counters (the reference keeps them in globals, src/variables.cpp:9-17); each
    // handle contributes the methods it ran before it is destroyed
    long long counts[DDAMG_COUNT_KINDS], hc[DDAMG_COUNT_KINDS];
    std::fill(counts, counts + DDAMG_COUNT_KINDS, -1LL);
    auto collect = [&]() {
        CHECK(ddamg_get_counters(h, hc));
        for (int k = 0; k < DDAMG_COUNT_KINDS; k++)
            if (hc[k] >= 0) counts[k] = hc[k];
    };

    // FGMRES with the V-cycle, then with the K-cycle; each constructs (sets up) its hierarchy
    std::vector<double> xv(2 * n), xk(2 * n);
    for (int cycle = 0; cycle < 2; cycle++) {
        std::cout << "--------------FGMRES with AMG " << (cycle ? "K" : "V") << "-cycle--------------" << std::endl;
        collect();
        ddamg_destroy(h);
        p.cycle = cycle ? DDAMG_CYCLE_K : DDAMG_CYCLE_V;
        CHECK(ddamg_create(&p, &h));
        CHECK(ddamg_load_gauge(h, U.data()));
        t0 = now();
        CHECK(ddamg_setup(h, 1));  // srand(rank2d + 1) of src/main.cpp:66
        std::vector<double>& xs = cycle ? xk : xv;
        st = ddamg_solve(h, b.data(), xs.data(), 1, &info);
        if (st != DDAMG_OK && st != DDAMG_NOT_CONVERGED) die("ddamg_solve", st);
        std::printf("FGMRES %s in %d iterations, relative residual %.3e\n",
                    info.converged ? "converged" : "did not converge", info.iterations, info.rel_residual);
        std::printf("time elapsed FGMRES AMG %c-cycle: %.4fs (setup %.4fs).\n\n", cycle ? 'K' : 'V', now() - t0,
                    info.setup_seconds);
    }
    collect();
    // src/main.cpp:89-97: check each solution, then write its metadata file (writeMetadata, src/io.cpp:72-145)
    std::cout << "Checking solution of V-cycle" << std::endl;
    check_solution(h, xv, b, Nt);
    CHECK(ddamg_write_metadata_params(&p, counts, 0, tol, nullptr));
    std::cout << "Checking solution of K-cycle" << std::endl;
    check_solution(h, xk, b, Nt);
    CHECK(ddamg_write_metadata_params(&p, counts, 1, tol, nullptr));
    if (argc > 3) CHECK(ddamg_write_binary(argv[3], Nx, Nt, xv.data()));
    ddamg_destroy(h);
    return 0;
}
