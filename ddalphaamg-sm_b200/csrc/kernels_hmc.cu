// Hybrid Monte Carlo for the two-flavour Schwinger model: the upstream producer of the gauge fields
// the solver consumes (the reference reads externally generated HMC configurations).  The action is
// S = beta sum_P (1 - cos theta_P) + phi^dagger (D^dagger D)^-1 phi, with the plaquette angle
// theta_P(x,t) = th0(x,t) + th1(x,t+1) - th0(x+1,t) - th1(x,t) (the convention of the Metropolis
// generator) and th[site*2 + mu] the angle of U_mu = exp(i th).  These kernels are the per-link pieces
// of the leapfrog integrator; the fermion force comes from the link-derivative kernel and
// U = exp(i theta) from theta_to_links_kernel (kernels_fine.cu).
#include "internal.h"

namespace ddamg {

__device__ __forceinline__ double plaq(const double* __restrict__ th, int Nx, int Nt, int x, int t) {
    const int n = x * Nt + t;
    const int ntp = x * Nt + ((t + 1 == Nt) ? 0 : t + 1);
    const int nxp = ((x + 1 == Nx) ? 0 : x + 1) * Nt + t;
    return th[2 * n] + th[2 * ntp + 1] - th[2 * nxp] - th[2 * n + 1];
}

// dS_g / d theta_mu(x) = beta sum over the two plaquettes holding the link of sin(theta_P) times the
// link's orientation in them: mu = 0 is +1 in P(x,t) and -1 in P(x-1,t); mu = 1 is -1 in P(x,t) and
// +1 in P(x,t-1)
__global__ void gauge_force_kernel(const double* __restrict__ th, double* __restrict__ F, int Nx, int Nt,
                                   double beta) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Nx * Nt) return;
    const int x = n / Nt, t = n - x * Nt;
    const double sp = sin(plaq(th, Nx, Nt, x, t));
    const double sxm = sin(plaq(th, Nx, Nt, (x == 0) ? Nx - 1 : x - 1, t));
    const double stm = sin(plaq(th, Nx, Nt, x, (t == 0) ? Nt - 1 : t - 1));
    F[2 * n] = beta * (sp - sxm);
    F[2 * n + 1] = beta * (stm - sp);
}

// p -= eps (F_gauge + 2 F_link), where F_link = -Re[(D X)^dagger dD/dtheta X] is the link-derivative
// kernel's output for psi = X, lambda = D X, and dS_f/dtheta = 2 F_link
__global__ void hmc_momentum_kernel(double* __restrict__ p, const double* __restrict__ Fg,
                                    const double* __restrict__ Ff, double eps, long nlinks) {
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nlinks) return;
    p[e] -= eps * (Fg[e] + 2.0 * Ff[e]);
}

// theta += eps p
__global__ void hmc_theta_kernel(double* __restrict__ th, const double* __restrict__ p, double eps, long nlinks) {
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nlinks) return;
    th[e] += eps * p[e];
}

void launch_gauge_force(cudaStream_t s, const double* th, double* F, int Nx, int Nt, double beta) {
    DDAMG_LAUNCH(gauge_force_kernel, ceil_div((long)Nx * Nt, 256), 256, 0, s, th, F, Nx, Nt, beta);
}
void launch_hmc_momentum(cudaStream_t s, double* p, const double* Fg, const double* Ff, double eps, long nlinks) {
    DDAMG_LAUNCH(hmc_momentum_kernel, ceil_div(nlinks, 256), 256, 0, s, p, Fg, Ff, eps, nlinks);
}
void launch_hmc_theta(cudaStream_t s, double* th, const double* p, double eps, long nlinks) {
    DDAMG_LAUNCH(hmc_theta_kernel, ceil_div(nlinks, 256), 256, 0, s, th, p, eps, nlinks);
}

}  // namespace ddamg
