/*
 * Harness main for the reference DD-alphaAMG (Schwinger model) sources, run as
 * one rank through oracle/ref_shim/mpi.h.  Test infrastructure only: its
 * outputs pin the CPU restatement (oracle/ddamg_oracle.c) and give the timed
 * CPU baseline.  It replaces the reference's stdin main (src/main.cpp) with
 * command-line arguments and fixes its single-rank init order
 * (src/main.cpp:61-62 sizes lpb/rpb before assignWidth()).
 *
 * Usage:
 *   ref_harness ops   <levels> <m0> <params> <conf.bin> <probe.bin> <tvec.bin> <outdir>
 *   ref_harness solve <levels> <m0> <params> <conf.bin> <rhs.bin> <tvec.bin|-> <outdir>
 *                     <cycle:0=V,1=K> <fgmres_m> <fgmres_restarts> <tol>
 *   ref_harness krylov <levels> <m0> <params> <conf.bin> <rhs.bin> <x0.bin|-> <outdir> <max_iter> <tol>
 *                     (bi_cgstab from x0, then Methods::CG: conjugate_gradient on D^dagger rhs)
 *   ref_harness multilevel <levels> <m0> <params> <conf.bin> <rhs.bin> <tvec.bin> <outdir> <cycle> <it> <tol>
 *                     (AlgebraicMG::applyMultilevel after the injected setup; prints its cycle count)
 *   ref_harness fgmres_sap <levels> <m0> <params> <conf.bin> <rhs.bin> - <outdir> <m> <restarts> <tol>
 *   ref_harness sapfine <levels> <m0> <params> <conf.bin> <rhs.bin> - <outdir> <xblocks> <tblocks> <nu>
 *   ref_harness metadata <levels> <m0> <params> <conf.bin> - - <outdir> <cycle> <tol>
 *                     <CG> <BiCG> <GMRES> <SAP> <FGMRES_SAP> <Vcycle> <Kcycle>
 *                     (writeMetadata with the iteration counters given; the file lands in outdir)
 *
 * conf.bin / rhs.bin use the reference binary record format (src/io.cpp:32-44).
 * probe.bin / tvec.bin / outputs are raw little-endian complex128 arrays
 * without halo, site index x*Nt+t, dof fastest (dof = c*2+alpha).
 * tvec.bin holds every random vector the setup consumes, in the order
 * AlgebraicMG::setUpPhase (src/amg.cpp:12-41) draws them; "-" uses the
 * reference's own mt19937 setup instead.
 */
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <random>
#include <sstream>
#include <string>
#include <vector>
#include <utility>
#include <unistd.h>

#define private public
#include "amg.h"
#include "conjugate_gradient.h"
#include "params.h"
#include "io.h"
#undef private

static std::string g_out;

static void dump(const std::string& name, const std::vector<c_double>& v) {
    std::ofstream f(g_out + "/" + name, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), v.size() * sizeof(c_double));
}

/* interior of a halo spinor -> compact [site][dof] */
static std::vector<c_double> interior(const spinor& s, int Nx, int Nt, int dof) {
    std::vector<c_double> out((size_t)Nx * Nt * dof);
    for (int x = 1; x <= Nx; x++)
        for (int t = 1; t <= Nt; t++)
            for (int d = 0; d < dof; d++)
                out[((size_t)(x - 1) * Nt + (t - 1)) * dof + d] = s.val[(x * (Nt + 2) + t) * dof + d];
    return out;
}
static void fill_interior(spinor& s, const c_double* src, int Nx, int Nt, int dof) {
    for (int x = 1; x <= Nx; x++)
        for (int t = 1; t <= Nt; t++)
            for (int d = 0; d < dof; d++)
                s.val[(x * (Nt + 2) + t) * dof + d] = src[((size_t)(x - 1) * Nt + (t - 1)) * dof + d];
}

struct Stream {
    std::vector<c_double> data;
    size_t pos = 0;
    void load(const std::string& path) {
        std::ifstream f(path, std::ios::binary | std::ios::ate);
        if (!f) { std::cerr << "cannot open " << path << "\n"; std::exit(3); }
        size_t n = f.tellg();
        f.seekg(0);
        data.resize(n / sizeof(c_double));
        f.read(reinterpret_cast<char*>(data.data()), n);
    }
    const c_double* take(size_t n) {
        if (pos + n > data.size()) { std::cerr << "vector stream too short\n"; std::exit(3); }
        const c_double* p = data.data() + pos;
        pos += n;
        return p;
    }
};

/* AlgebraicMG::setUpPhase (src/amg.cpp:4-56) with the random draws taken from a stream */
static void setup_injected(AlgebraicMG& amg, Stream& rnd) {
    auto& L = amg.levels;
    for (int cc = 0; cc < L[0]->Ntest; cc++)
        fill_interior(L[0]->tvec[cc], rnd.take((size_t)L[0]->Nx * L[0]->Nt * L[0]->DOF), L[0]->Nx, L[0]->Nt, L[0]->DOF);
    for (int l = 1; l < LevelV::levels - 1; l++)
        for (int cc = 0; cc < L[l]->Ntest; cc++) {
            if (cc < L[l - 1]->Ntest)
                L[l - 1]->Pdagg_v(L[l - 1]->tvec[cc], L[l]->tvec[cc]);
            else
                fill_interior(L[l]->tvec[cc], rnd.take((size_t)L[l]->Nx * L[l]->Nt * L[l]->DOF), L[l]->Nx, L[l]->Nt,
                              L[l]->DOF);
        }
    for (int l = 0; l < LevelV::levels - 1; l++) {
        spinor rhs((L[l]->Nt + 2) * (L[l]->Nx + 2) * L[l]->DOF);
        for (int cc = 0; cc < L[l]->Ntest; cc++)
            L[l]->sap_l->SAP(rhs, L[l]->tvec[cc], AMGV::SAP_test_vectors_iterations, 1e-10, false);
        L[l]->orthonormalize();
        L[l]->makeCoarseLinks(*L[l + 1]);
    }
}

/* outer solver: FGMRES_AMG (include/amg.h:147-270) with the cycle chosen at run time */
class HarnessFGMRES : public FGMRES {
   public:
    HarnessFGMRES(AlgebraicMG& amg, const spinor& U, double m0, int cycle, int m, int restarts, double tol)
        : FGMRES(LV::Ntot, LV::dof, mpi::maxSizeH, 1, 1, mpi::width_x, mpi::width_t, m, restarts, tol),
          amg(amg), U(U), m0(m0), cycle(cycle) {}
    AlgebraicMG& amg;
    const spinor& U;
    double m0;
    int cycle;
    void func(const spinor& in, spinor& out) override { D_phi(U, in, out, m0); }
    void preconditioner(const spinor& in, spinor& out) override {
        for (int i = 0; i < mpi::maxSizeH; i++) out.val[i] = 0;
        if (cycle == 0) amg.v_cycle(0, in, out);
        else amg.k_cycle(0, in, out);
    }
    c_double dot(c_double* A, c_double* B) override { return ::dot(A, B); }
    void axpy(const spinor& X, const spinor& Y, const c_double& lambda, spinor& out) override {
        ::axpy(X, Y, lambda, out);
    }
    void scal(const c_double& lambda, const spinor& X, spinor& Y) override { ::scal(lambda, X, Y); }
};

static double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int main(int argc, char** argv) {
    if (argc < 9) {
        std::cerr << "usage: see header\n";
        return 2;
    }
    std::string mode = argv[1];
    LevelV::levels = std::atoi(argv[2]);
    double m0 = std::atof(argv[3]);
    std::string pfile = argv[4], conf = argv[5], vfile = argv[6], tfile = argv[7];
    g_out = argv[8];
    mass::m0 = m0;
    mpi::size = 1;
    mpi::rank = 0;
    mpi::ranks_x = 1;
    mpi::ranks_t = 1;
    LevelV::maxLevel = LevelV::levels - 1;
    assignWidth();  /* must precede allocate_lattice_arrays with one rank */
    allocate_lattice_arrays();
    initializeMPI();
    readParameters(pfile);
    boundaries();

    spinor U(mpi::maxSizeH);
    read_binary(conf, U);

    if (mode == "ops") {
        Stream probe, rnd;
        probe.load(vfile);
        rnd.load(tfile);
        AlgebraicMG amg(U, m0, AMGV::nu1, AMGV::nu2);
        setup_injected(amg, rnd);
        auto& L = amg.levels;
        std::vector<spinor> pr;
        for (int l = 0; l < LevelV::levels; l++) {
            spinor s((L[l]->Nx + 2) * (L[l]->Nt + 2) * L[l]->DOF);
            fill_interior(s, probe.take((size_t)L[l]->Nx * L[l]->Nt * L[l]->DOF), L[l]->Nx, L[l]->Nt, L[l]->DOF);
            pr.push_back(s);
        }
        /* fine operators (src/dirac_operator.cpp:24-85) */
        {
            spinor o(mpi::maxSizeH);
            D_phi(U, pr[0], o, m0);
            dump("Dphi.bin", interior(o, L[0]->Nx, L[0]->Nt, 2));
            D_dagger_phi(U, pr[0], o, m0);
            dump("Ddagphi.bin", interior(o, L[0]->Nx, L[0]->Nt, 2));
        }
        for (int l = 0; l < LevelV::levels; l++) {
            Level& lv = *L[l];
            int n = lv.Nx, t = lv.Nt, d = lv.DOF;
            std::string sl = std::to_string(l);
            spinor o((n + 2) * (t + 2) * d);
            lv.D_operator(pr[l], o);
            dump("Dop_" + sl + ".bin", interior(o, n, t, d));
            if (l >= 1) {
                /* coarse links as built by makeCoarseLinks of level l-1 (src/level.cpp:431-542) */
                int C = lv.colors;
                std::vector<c_double> g1((size_t)n * t * 4 * C * C), g2((size_t)n * t * 8 * C * C),
                    g3((size_t)n * t * 8 * C * C);
                for (int x = 1; x <= n; x++)
                    for (int tt = 1; tt <= t; tt++) {
                        int h = x * (t + 2) + tt;
                        size_t s = (size_t)(x - 1) * t + (tt - 1);
                        for (int k = 0; k < 4 * C * C; k++) g1[s * 4 * C * C + k] = lv.G1.val[(size_t)h * 4 * C * C + k];
                        for (int k = 0; k < 8 * C * C; k++) {
                            g2[s * 8 * C * C + k] = lv.G2.val[(size_t)h * 8 * C * C + k];
                            g3[s * 8 * C * C + k] = lv.G3.val[(size_t)h * 8 * C * C + k];
                        }
                    }
                dump("G1_" + sl + ".bin", g1);
                dump("G2_" + sl + ".bin", g2);
                dump("G3_" + sl + ".bin", g3);
            }
            if (l < LevelV::maxLevel) {
                std::vector<c_double> tv;
                for (int cc = 0; cc < lv.Ntest; cc++) {
                    auto v = interior(lv.tvec[cc], n, t, d);
                    tv.insert(tv.end(), v.begin(), v.end());
                }
                dump("tvec_" + sl + ".bin", tv);
                Level& nx = *L[l + 1];
                spinor c((nx.Nx + 2) * (nx.Nt + 2) * nx.DOF);
                lv.Pdagg_v(pr[l], c);
                dump("Pdagg_" + sl + ".bin", interior(c, nx.Nx, nx.Nt, nx.DOF));
                lv.P_vc(pr[l + 1], o);
                dump("P_" + sl + ".bin", interior(o, n, t, d));
                /* SAP_C::SAP (src/sap.cpp:81-165), nu = 3 from x = 0 */
                spinor xs((n + 2) * (t + 2) * d);
                int it = lv.sap_l->SAP(pr[l], xs, 3, 1e-10, false);
                dump("SAP_" + sl + ".bin", interior(xs, n, t, d));
                std::ofstream(g_out + "/SAP_" + sl + ".txt") << it << "\n";
            } else {
                /* coarsest GMRES (include/level.h:70-140), x0 = rhs */
                spinor xs((n + 2) * (t + 2) * d);
                int it = lv.gmres_l->fgmres(pr[l], pr[l], xs, false);
                dump("coarse_gmres.bin", interior(xs, n, t, d));
                std::ofstream(g_out + "/coarse_gmres.txt") << it << "\n";
            }
        }
        {
            spinor psi(mpi::maxSizeH);
            amg.v_cycle(0, pr[0], psi);
            dump("vcycle.bin", interior(psi, L[0]->Nx, L[0]->Nt, 2));
            spinor psk(mpi::maxSizeH);
            amg.k_cycle(0, pr[0], psk);
            dump("kcycle.bin", interior(psk, L[0]->Nx, L[0]->Nt, 2));
        }
        return 0;
    }

    if (mode == "solve") {
        if (argc < 13) {
            std::cerr << "solve needs cycle m restarts tol\n";
            return 2;
        }
        int cycle = std::atoi(argv[9]);
        FGMRESV::fgmres_restart_length = std::atoi(argv[10]);
        FGMRESV::fgmres_restarts = std::atoi(argv[11]);
        double tol = std::atof(argv[12]);
        spinor rhs(mpi::maxSizeH), x0(mpi::maxSizeH), x(mpi::maxSizeH);
        read_binary(vfile, rhs);
        double t0 = now();
        AlgebraicMG amg(U, m0, AMGV::nu1, AMGV::nu2);
        if (tfile == "-") {
            amg.setUpPhase(AMGV::Nit);
        } else {
            Stream rnd;
            rnd.load(tfile);
            setup_injected(amg, rnd);
        }
        double t1 = now();
        HarnessFGMRES solver(amg, U, m0, cycle, FGMRESV::fgmres_restart_length, FGMRESV::fgmres_restarts, tol);
        int iters = solver.fgmres(rhs, x0, x, false);
        double t2 = now();
        /* true relative residual with D_phi */
        spinor r(mpi::maxSizeH);
        D_phi(U, x, r, m0);
        double nr = 0, nb = 0;
        for (int xx = 1; xx <= mpi::width_x; xx++)
            for (int tt = 1; tt <= mpi::width_t; tt++)
                for (int mu = 0; mu < 2; mu++) {
                    int i = idx(xx, tt, mu);
                    nr += std::norm(r.val[i] - rhs.val[i]);
                    nb += std::norm(rhs.val[i]);
                }
        dump("x.bin", interior(x, mpi::width_x, mpi::width_t, 2));
        std::ofstream m(g_out + "/solve.txt");
        m.precision(17);
        m << "iterations " << iters << "\nsetup_s " << (t1 - t0) << "\nsolve_s " << (t2 - t1) << "\nrelres "
          << std::sqrt(nr / nb) << "\n";
        return 0;
    }
    if (mode == "multilevel") {
        /* AlgebraicMG::applyMultilevel (src/amg.cpp:177-243) after an injected setup; it prints the
         * cycle count itself ("V-cycle converged in N cycles"), which the caller reads from stdout */
        if (argc < 12) {
            std::cerr << "multilevel needs cycle it tol\n";
            return 2;
        }
        AMGV::cycle = std::atoi(argv[9]);
        const int it = std::atoi(argv[10]);
        const double tol = std::atof(argv[11]);
        spinor rhs(mpi::maxSizeH), x(mpi::maxSizeH);
        read_binary(vfile, rhs);
        AlgebraicMG amg(U, m0, AMGV::nu1, AMGV::nu2);
        Stream rnd;
        rnd.load(tfile);
        setup_injected(amg, rnd);
        amg.applyMultilevel(it, rhs, x, tol, true);
        dump("x.bin", interior(x, mpi::width_x, mpi::width_t, 2));
        return 0;
    }
    if (mode == "fgmres_sap") {
        /* FGMRES_SAP (include/sap.h:236-333) as Methods::FGMRES_sap builds it (src/methods.cpp:83-104) */
        if (argc < 12) {
            std::cerr << "fgmres_sap needs m restarts tol\n";
            return 2;
        }
        const int len = std::atoi(argv[9]), restarts = std::atoi(argv[10]);
        const double tol = std::atof(argv[11]);
        spinor rhs(mpi::maxSizeH), x0(mpi::maxSizeH), x(mpi::maxSizeH);
        read_binary(vfile, rhs);
        FGMRES_SAP fs(LV::Ntot, LV::dof, mpi::maxSizeH, 1, 1, mpi::width_x, mpi::width_t, len, restarts, tol, U, m0);
        const int iters = fs.fgmres(rhs, x0, x, false);
        dump("x.bin", interior(x, mpi::width_x, mpi::width_t, 2));
        std::ofstream(g_out + "/fgmres_sap.txt") << "iterations " << iters << "\n";
        return 0;
    }
    if (mode == "sapfine") {
        /* Methods::SAP (src/methods.cpp:60-80): SAP_fine_level over xblocks x tblocks, from x = 0 */
        if (argc < 12) {
            std::cerr << "sapfine needs xblocks tblocks nu\n";
            return 2;
        }
        const int xb = std::atoi(argv[9]), tb = std::atoi(argv[10]), nu = std::atoi(argv[11]);
        spinor rhs(mpi::maxSizeH), x(mpi::maxSizeH);
        read_binary(vfile, rhs);
        SAP_fine_level sap(mpi::width_x, mpi::width_t, xb, tb, 2, 1);
        sap.set_params(U, m0);
        const int it = sap.SAP(rhs, x, nu, 1e-10, false);
        dump("x.bin", interior(x, mpi::width_x, mpi::width_t, 2));
        std::ofstream(g_out + "/sapfine.txt") << "iterations " << it << "\n";
        return 0;
    }
    if (mode == "metadata") {
        /* writeMetadata (src/io.cpp:72-145) with the iteration counters set from the command line;
         * the FLOP counters keep their initial -1 */
        if (argc < 18) {
            std::cerr << "metadata needs cycle tol and 7 counters\n";
            return 2;
        }
        const int cycle = std::atoi(argv[9]);
        const double tol = std::atof(argv[10]);
        iter_counters::CGIt = std::atoll(argv[11]);
        iter_counters::BiCGIt = std::atoll(argv[12]);
        iter_counters::GMRESIt = std::atoll(argv[13]);
        iter_counters::SAPIt = std::atoll(argv[14]);
        iter_counters::FGMRES_SAPIt = std::atoll(argv[15]);
        iter_counters::vCycleIt = std::atoll(argv[16]);
        iter_counters::kCycleIt = std::atoll(argv[17]);
        setenv("HOSTNAME", "golden-host", 1);
        if (chdir(g_out.c_str()) != 0) return 3;
        writeMetadata(cycle, tol);
        return 0;
    }
    if (mode == "krylov") {
        if (argc < 11) {
            std::cerr << "krylov needs max_iter tol\n";
            return 2;
        }
        const int max_iter = std::atoi(argv[9]);
        const double tol = std::atof(argv[10]);
        spinor rhs(mpi::maxSizeH), x0(mpi::maxSizeH), xb(mpi::maxSizeH), xc(mpi::maxSizeH), ddag(mpi::maxSizeH);
        read_binary(vfile, rhs);
        if (tfile != "-") {
            Stream s0;
            s0.load(tfile);
            fill_interior(x0, s0.take((size_t)mpi::width_x * mpi::width_t * 2), mpi::width_x, mpi::width_t, 2);
        }
        BiCG::max_iter = max_iter;
        BiCG::tol = tol;
        CG::max_iter = max_iter;
        CG::tol = tol;
        double t0 = now();
        int itb = bi_cgstab(U, rhs, x0, xb, m0, false);
        double t1 = now();
        D_dagger_phi(U, rhs, ddag, m0);  /* Methods::CG (src/methods.cpp:42-58) */
        double t2 = now();
        int itc = conjugate_gradient(U, ddag, xc, m0, false);
        double t3 = now();
        dump("x_bicg.bin", interior(xb, mpi::width_x, mpi::width_t, 2));
        dump("x_cg.bin", interior(xc, mpi::width_x, mpi::width_t, 2));
        std::ofstream m(g_out + "/krylov.txt");
        m.precision(17);
        m << "bicg_iterations " << itb << "\nbicg_s " << (t1 - t0) << "\ncg_iterations " << itc << "\ncg_s "
          << (t3 - t2) << "\n";
        return 0;
    }
    std::cerr << "unknown mode " << mode << "\n";
    return 2;
}
