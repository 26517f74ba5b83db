// Direct pairwise D3(BJ) lattice sum on the device (float64): the continuum tail beyond the
// pair cutoff, the chain of dE/dc to dE/dCN, and the final energy and stress. The pair kernel
// itself is k_direct_pairs (cell-list traversal, fd3_cells.cu). The restatement it follows is
// the oracle's direct sum: E = -1/2 sum'_{i,j,n} C6_ij phi_XY(r) within r_direct, plus
//   E_tail = -(2 pi / Omega) sum_r lambda_r sum_XY A_X^r A_Y^r I_XY,  A_X^r = sum_{i in X} c_ir,
//   I_XY = int_Rc^inf r^2 phi_XY(r) dr   (r^-6 part in closed form, r^-8 part as a series in
//   (R0/Rc)^8), dE_tail/dc_ir = -(4 pi / Omega) lambda_r sum_Y I_XY A_Y^r, and the tail virial
//   (-E_tail + (2 pi Rc^3 / (3 Omega)) sum_r lambda_r sum_XY A A phi_XY(Rc)) on the diagonal.
// The physics constants follow src/fourierd3/pair_pot.py:55-105 (R0_XY, qq = sqrt(Q_X Q_Y)).
#include "fd3_internal.h"

namespace fd3 {

constexpr int kDirThreads = 256;

// Per-block partial sums of c_ir per (species X, rank r): thread (X, r) walks the block's atom
// range in order (fixed summation order, no atomics). part[b * S * R + X * R + r].
__global__ void __launch_bounds__(kDirThreads) k_direct_species_sums(int n, int per_block,
                                                                    const int32_t* __restrict__ species,
                                                                    const double* __restrict__ c6, int S, int R,
                                                                    double* __restrict__ part) {
  const int a0 = blockIdx.x * per_block;
  const int a1 = a0 + per_block < n ? a0 + per_block : n;
  for (int e = threadIdx.x; e < S * R; e += blockDim.x) {
    const int X = e / R, r = e - X * R;
    double s = 0.0;
    for (int i = a0; i < a1; ++i)
      if (species[i] == X) s += c6[(size_t)i * R + r];
    part[(size_t)blockIdx.x * S * R + e] = s;
  }
}

// One block: A (fixed-order sum of the partials), the tail integrals I_XY and phi_XY(Rc), the
// tail energy and virial scalar (tail[0], tail[1]) and T_Xr = -(4 pi / Omega) lambda_r sum_Y
// I_XY A_Y^r (the tail's dE/dc of an atom of species X).
__global__ void __launch_bounds__(kDirThreads) k_direct_tail(int nb, const double* __restrict__ part, int S, int R,
                                                            const Tables* __restrict__ tab,
                                                            const GreenPair* __restrict__ gp, double rc,
                                                            const CellInfo* __restrict__ ci,
                                                            double* __restrict__ A, double* __restrict__ tail,
                                                            double* __restrict__ T) {
  const int SR = S * R;
  for (int e = threadIdx.x; e < SR; e += blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += part[(size_t)b * SR + e];
    A[e] = s;
  }
  const double s6 = tab->s6, s8 = tab->s8, kPi_ = 3.14159265358979323846;
  const double vol = ci->volume;
  // I_XY and phi_XY(Rc) in the scratch after T (2 S^2 values)
  double* I = T + SR;
  double* phiR = I + S * S;
  for (int e = threadIdx.x; e < S * S; e += blockDim.x) {
    const GreenPair q = gp[e];
    const double a3 = q.R * q.R * q.R;
    const double i6 = (0.5 * kPi_ - atan(rc * rc * rc / a3)) / (3.0 * a3);
    const double t = pow(q.R / rc, 8.0);
    double i8 = 0.0, term = pow(rc, -5.0);
    for (int k = 0; k < 12; ++k) {
      i8 += ((k & 1) ? -term : term) / (5.0 + 8.0 * k);
      term *= t;
    }
    I[e] = s6 * i6 + 3.0 * s8 * q.qq * i8;
    const double R02 = q.R * q.R, R06 = R02 * R02 * R02, R08 = R06 * R02;
    const double rc6 = rc * rc * rc * rc * rc * rc;
    phiR[e] = s6 / (rc6 + R06) + 3.0 * s8 * q.qq / (rc6 * rc * rc + R08);
  }
  __syncthreads();
  for (int e = threadIdx.x; e < SR; e += blockDim.x) {
    const int X = e / R, r = e - X * R;
    double s = 0.0;
    for (int Y = 0; Y < S; ++Y) s += I[X * S + Y] * A[Y * R + r];
    T[e] = -(4.0 * kPi_ / vol) * tab->eigs[r] * s;
  }
  if (threadIdx.x == 0) {
    double et = 0.0, su = 0.0;
    for (int r = 0; r < R; ++r)
      for (int X = 0; X < S; ++X)
        for (int Y = 0; Y < S; ++Y) {
          const double aa = tab->eigs[r] * A[X * R + r] * A[Y * R + r];
          et += aa * I[X * S + Y];
          su += aa * phiR[X * S + Y];
        }
    et *= -(2.0 * kPi_ / vol);
    su *= 2.0 * kPi_ * rc * rc * rc / (3.0 * vol);
    tail[0] = et;
    tail[1] = -et + su;
  }
}

// dE/dCN_i = sum_r (dE/dc_ir + T_{X_i r}) dc_ir/dCN_i
__global__ void __launch_bounds__(kDirThreads) k_direct_gcn(int n, const int32_t* __restrict__ species,
                                                           const double* __restrict__ dEdc,
                                                           const double* __restrict__ T, const double* __restrict__ dc6,
                                                           int R, double* __restrict__ gcn) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int X = species[i];
  double g = 0.0;
  for (int r = 0; r < R; ++r) g += (dEdc[(size_t)i * R + r] + T[X * R + r]) * dc6[(size_t)i * R + r];
  gcn[i] = g;
}

// E [eV] = (-1/2 sum e + E_tail) and stress [eV/A^3] = (W_pair + W_tail I + W_cn) / Omega
__global__ void __launch_bounds__(256) k_direct_finalize(const double* __restrict__ pair_part, int n_pair,
                                                         const double* __restrict__ tail,
                                                         const double* __restrict__ cnv_part, int n_cnv,
                                                         const CellInfo* __restrict__ ci, double* __restrict__ energy,
                                                         double* __restrict__ stress) {
  double v[16];
  for (int k = 0; k < 16; ++k) v[k] = 0.0;
  for (int b = threadIdx.x; b < n_pair; b += blockDim.x)
    for (int c = 0; c < 7; ++c) v[c] += pair_part[7 * b + c];
  for (int b = threadIdx.x; b < n_cnv; b += blockDim.x)
    for (int c = 0; c < 9; ++c) v[7 + c] += cnv_part[9 * b + c];
  __shared__ double tot[16];
  block_sum_store<16>(v, tot);
  if (threadIdx.x != 0) return;
  const double vol = ci->volume;
  *energy = (-0.5 * tot[0] + tail[0]) * kHartreeToEv;
  const double W[9] = {tot[1], tot[2], tot[3], tot[2], tot[4], tot[5], tot[3], tot[5], tot[6]};
  const double a2b3 = kAngToBohr * kAngToBohr * kAngToBohr;
  for (int k = 0; k < 9; ++k) {
    const double wt = (k == 0 || k == 4 || k == 8) ? tail[1] : 0.0;
    stress[k] = (W[k] + wt + tot[7 + k]) * kHartreeToEv / vol * a2b3;
  }
}

size_t direct_scratch_doubles(int S, int R) { return (size_t)S * R + 2 * (size_t)S * S; }

int launch_direct_tail_gcn(int n, const int32_t* species, const double* c6, const double* dc6, const double* dEdc,
                           const Tables* tab, const GreenPair* gp, int S, int R, double rc_bohr, const CellInfo* ci,
                           double* sp_part, int sp_blocks, double* A, double* tail, double* T, double* gcn,
                           cudaStream_t s) {
  const int per = (n + sp_blocks - 1) / sp_blocks;
  k_direct_species_sums<<<sp_blocks, kDirThreads, 0, s>>>(n, per, species, c6, S, R, sp_part);
  FD3_LAUNCHED();
  k_direct_tail<<<1, kDirThreads, 0, s>>>(sp_blocks, sp_part, S, R, tab, gp, rc_bohr, ci, A, tail, T);
  FD3_LAUNCHED();
  k_direct_gcn<<<(n + kDirThreads - 1) / kDirThreads, kDirThreads, 0, s>>>(n, species, dEdc, T, dc6, R, gcn);
  FD3_LAUNCHED();
  return FD3_OK;
}

int launch_direct_finalize(const double* pair_part, int n_pair, const double* tail, const double* cnv_part, int n_cnv,
                           const CellInfo* ci, double* energy, double* stress, cudaStream_t s) {
  k_direct_finalize<<<1, 256, 0, s>>>(pair_part, n_pair, tail, cnv_part, n_cnv, ci, energy, stress);
  FD3_LAUNCHED();
  return FD3_OK;
}

}  // namespace fd3
