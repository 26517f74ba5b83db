/*
 * fd3.h -- C ABI of the B200 FourierD3 dispersion library (libfd3.so).
 *
 * The library evaluates the DFT-D3(BJ) dispersion energy of a 3D-periodic box in
 * reciprocal space from a low-rank C6 decomposition, together with its exact
 * derivatives (forces, cell gradient / virial), on one NVIDIA B200 (sm_100a).
 *
 * Conventions
 *   - Every pointer argument named d_* is DEVICE memory owned by the caller; h_* is
 *     host memory. No function allocates device memory except fd3_plan_create (small
 *     per-species tables and cuFFT plan handles). All large scratch lives in a caller
 *     supplied workspace whose size fd3_workspace_size returns.
 *   - Work is stream-ordered on the caller's stream; nothing synchronises the host
 *     except fd3_neighbor_count (returns the edge count) and fd3_plan_create.
 *   - Internal length unit Bohr (1 A = 1/0.52917726 Bohr), energy unit Hartree,
 *     except where an argument says Angstrom.
 *   - Status codes: FD3_OK on success; no C++ exception crosses this boundary.
 *   - A plan is not thread-safe; use one plan per stream.
 */
#ifndef FD3_H
#define FD3_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FD3_API __attribute__((visibility("default")))
#else
#define FD3_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  FD3_OK = 0,
  FD3_EINVAL = 1,     /* bad argument (shape, range, unsupported option)          */
  FD3_ECAPACITY = 2,  /* output capacity too small; the needed size is written back */
  FD3_ECUDA = 3,      /* a CUDA runtime call failed                               */
  FD3_ECUFFT = 4,     /* a cuFFT call failed                                      */
  FD3_ENOMEM = 5,     /* workspace smaller than fd3_workspace_size                */
} fd3_status;

enum { FD3_METHOD_SPME = 0, FD3_METHOD_PME = 1, FD3_METHOD_EWALD = 2 };
enum { FD3_PREC_FP64 = 0, FD3_PREC_MIXED = 1 };

typedef struct fd3_plan fd3_plan;

/* Everything the reference fixes at model construction (src/fourierd3/core.py:50-242).
 * Table arrays are host pointers, copied by fd3_plan_create. */
typedef struct {
  int32_t n_species;      /* S: unique elements present                           */
  int32_t n_rank;         /* r: rank of the C6 decomposition (utils.py:35-73)      */
  int32_t method;         /* FD3_METHOD_*  (core.py:184-242)                       */
  int32_t order;          /* p: interpolation nodes per axis, 1..8 (spme / pme)    */
  int32_t mesh[3];        /* nx, ny, nz (spme / pme; core.py:186)                  */
  int32_t ewald_ns[3];    /* Miller-index box (ewald; core.py:228-230)             */
  int32_t precision;      /* FD3_PREC_*                                            */
  int32_t has_cncorr;     /* 1: apply cncorr (core.py:383-384)                     */
  double r_cut;           /* CN cutoff in Bohr (core.py:121)                       */
  double params[4];       /* s6, s8, a1, a2 (core.py:165-170)                      */
  const double* rcov;     /* [S]      covalent radii, Bohr (core.py:152)           */
  const double* cnref;    /* [S*7]    reference CNs, -1 = unused (core.py:155)     */
  const double* eigvecs;  /* [S*7*r]  V reshaped (S, 7, r) (core.py:148)           */
  const double* eigs;     /* [r]      lambda (core.py:139-142)                     */
  const double* sqrtq;    /* [S]      sqrt(Q) (pair_pot.py:53)                     */
  const double* cncorr;   /* [S*2]    columns [b, a] or NULL                       */
  const float* deconv;    /* [nx*ny*(nz/2+1)] the float32 SPME window
                             sinc^(2p) clamped at 1e-10, exactly as the reference
                             builds it (pair_pot.py:180-207); NULL: evaluate it in
                             float64 inside the filter kernel instead            */
  int32_t cnfunc;         /* FD3_CN_SMOOTH (core.py:323-386, needs neighbours) or
                             FD3_CN_D4 (k-space D4 CN, core.py:388-447: spme/pme,
                             at most 8 species, no neighbour list; cncorr unused) */
  const double* rcov_cn;  /* [S] D4 CN covalent radii, Bohr (pair_pot.py:294); D4 */
  const double* en;       /* [S] electronegativities (pair_pot.py:301); D4 only   */
} fd3_plan_desc;
enum { FD3_CN_SMOOTH = 0, FD3_CN_D4 = 1 };

/* Replaces: FourierD3.__init__ buffers + KSpaceFilterD3 / MeshInterpolatorD3 /
 * D3Potential construction (src/fourierd3/core.py:50-242). */
FD3_API int fd3_plan_create(const fd3_plan_desc* desc, fd3_plan** out);
FD3_API int fd3_plan_destroy(fd3_plan* plan);

/* Launch-shape knobs an autotuner may set per plan (no reference counterpart: the
 * reference's torch ops choose their own launches). They change only how the work is
 * mapped onto the GPU; results agree with the defaults to rounding (a different
 * summation order), and every value is checked against the plan's sizes.
 *   FD3_TUNE_FILTER_KT  k-points per shared-memory tile of the reciprocal-space filter:
 *                       0 = per-thread register kernel (at most 8 species), 1, 2, 4, 8
 *                       or 16 = tiled kernel, -1 = the default for (species, rank).
 *   FD3_TUNE_SPREAD_ZC  z-tiles per column chunk of the mesh spread: 0 = one CTA per
 *                       16x16x8 tile, 1..64 = one CTA per 16x16 column chunk (capped by
 *                       the mesh), -1 = the default (8).
 *   FD3_TUNE_SPREAD_CAP staged atoms per column chunk at most: 0 = what shared memory
 *                       holds, >= 256 = a lower bound (denser chunks take the per-tile
 *                       staging path inside the same CTA).
 *   FD3_TUNE_FFT_X      1 = cuFFT transforms the (y, z) planes and one kernel does the x
 *                       transform, the filter and the inverse x transform per pencil (where
 *                       it applies: at most 4 species and 8 ranks, nx = 64, 128 or 256); 2 =
 *                       the same with units of rank groups moved by TMA (mixed precision); 0 =
 *                       3D cuFFT around a separate filter; -1 = the default (0). Which is
 *                       faster depends on the mesh and precision: time them.
 *   FD3_TUNE_XPENCIL    kz values per pencil of the fused x-pass: 1, 2 or 4 (used when the
 *                       pencil fits in shared memory), -1 = the default (the widest that
 *                       leaves three CTAs per SM for float, within 100 KB for double);
 *                       the value in effect is 0 where the fused x-pass does not apply.
 *   FD3_TUNE_XQ         TMA x-pass (FD3_TUNE_FFT_X = 2, mixed precision): flattened (y, kz)
 *                       values per unit, 4, 8, 16 or 32; -1 = the default (16).
 *   FD3_TUNE_XRANKS     TMA x-pass: ranks per unit, 1, 2 or 4; -1 = the default (1).
 *   FD3_TUNE_FILTER_MMA mixed precision, separate filter: 1 = the per-k-point S x S products
 *                       on the tensor cores (tcgen05.mma kind::tf32, operands split into tf32
 *                       high and low parts; at most 64 species and 8 ranks, as shared memory
 *                       allows), 0 or -1 = CUDA cores (the default).
 *   FD3_TUNE_GATHER_TILE fused-path gather: 1 = one CTA per (mesh tile, species) that stages
 *                       the tile's potential box once by TMA (at most 8 ranks, the box within
 *                       113 KB of shared memory); 0 or -1 (the default) = warp per atom reading
 *                       the mesh directly (faster unless a tile holds many atoms per species).
 *   FD3_TUNE_FFT_YZ     mixed precision with the fused x-pass (FD3_TUNE_FFT_X = 1 or 2) and
 *                       ny = nz = 256: 1 or 2 = the (y, z) plane transforms by this library's
 *                       cluster kernels (one pass over the mesh each way instead of cuFFT's
 *                       two; 1: clusters of 2 CTAs, one per SM; 2: the forward transform on
 *                       clusters of 4, two per SM); 0 = cuFFT; -1 = the default (1).
 * fd3_plan_get_tuning returns the value in effect (the default resolved). */
#define FD3_TUNE_FILTER_KT 0
#define FD3_TUNE_SPREAD_ZC 1
#define FD3_TUNE_SPREAD_CAP 2
#define FD3_TUNE_FFT_X 3
#define FD3_TUNE_XPENCIL 4
#define FD3_TUNE_XQ 5
#define FD3_TUNE_XRANKS 6
#define FD3_TUNE_FILTER_MMA 7
#define FD3_TUNE_GATHER_TILE 8
#define FD3_TUNE_FFT_YZ 9
FD3_API int fd3_plan_set_tuning(fd3_plan* plan, int32_t knob, int32_t value);
FD3_API int fd3_plan_get_tuning(const fd3_plan* plan, int32_t knob, int32_t* value);

/* Workspace bytes for a call with n_atoms atoms. n_bins: cell-list bins of the
 * fused path (0 for the edge path; see fd3_cell_grid). */
FD3_API int fd3_workspace_size(const fd3_plan* plan, int64_t n_atoms, int64_t n_bins, size_t* bytes);

/* Cell-list geometry for a box: bins per axis and the bin reach (A). */
FD3_API int fd3_cell_grid(const double* h_cell_ang, double r_cut_ang, int32_t* nbins3, int32_t* reach3);

/*
 * Energy and gradients from a caller-supplied edge list -- the reference's module
 * surface FourierD3.forward(positions, edge_index, shifts) (core.py:480-583) whose
 * autograd the reference relies on (calculator.py:177-188).
 *   d_pos      [N*3]  positions, Bohr
 *   d_species  [N]    compact species ids 0..S-1 (core.py:104-114)
 *   d_cell     [9]    cell rows, Bohr
 *   d_src,d_dst[E]    edge_index rows (int64)
 *   d_shift    [E*3]  Cartesian shift vectors, Bohr
 * outputs (any gradient pointer may be NULL when need_grad == 0):
 *   d_energy   [1]    energy, Hartree
 *   d_gpos     [N*3]  dE/dpos      (Hartree/Bohr)
 *   d_gshift   [E*3]  dE/dshift    (Hartree/Bohr)
 *   d_gcell    [9]    dE/dcell     (Hartree/Bohr), positions and shifts held fixed
 * The workspace is sized by fd3_edge_workspace_size (it holds the edges sorted by source and
 * by destination). Edges may come in any order; every per-atom sum is taken in edge order, so
 * repeated calls give bitwise-equal results. No host synchronisation: an edge index outside
 * 0..N-1 is not dereferenced, and it makes the energy and gradients NaN.
 */
FD3_API int fd3_edge_workspace_size(const fd3_plan* plan, int64_t n_atoms, int64_t n_edges, size_t* bytes);

/* Edge-list option (no reference counterpart; off by default, as in the reference, where every
 * edge passed to forward counts): on = 1 makes edges with |r| >= the CN cutoff contribute
 * nothing to the CN and its gradients, so an MD driver can pass its Verlet list (cutoff + skin)
 * unchanged between rebuilds -- a fixed edge count, which a captured CUDA graph needs --
 * instead of cutting it back to the cutoff before every call. */
FD3_API int fd3_plan_set_edge_cutoff(fd3_plan* plan, int32_t on);
FD3_API int fd3_energy_edges(fd3_plan* plan, int64_t n_atoms, const double* d_pos, const int32_t* d_species,
                     const double* d_cell, int64_t n_edges, const int64_t* d_src, const int64_t* d_dst,
                     const double* d_shift, int32_t need_grad, void* d_work, size_t work_bytes,
                     double* d_energy, double* d_gpos, double* d_gshift, double* d_gcell, void* stream);

/*
 * Fused energy + forces + stress with the neighbour search done on the device by a
 * cell list (no edge list is materialised) -- the ASE calculator path
 * FourierD3ASECalculator.calculate (calculator.py:125-192) including its matscipy
 * neighbour build (calculator.py:94-123).
 *   d_pos_ang [N*3]  positions, Angstrom;  h_cell_ang [9] cell rows, Angstrom (host)
 *   d_cell_ang [9]   the same cell on the device
 *   r_cut_ang        neighbour cutoff (the pair predicate uses Angstrom, as matscipy)
 * outputs: d_energy [1] eV, d_forces [N*3] eV/A, d_stress [9] eV/A^3 (ASE sign)
 * All work is ordered on `stream`; the mesh sort runs on the plan's own side stream, forked
 * from and joined back to `stream` by events (so one plan serialises the sorts of calls made
 * on different streams, and the call may be captured into a CUDA graph).
 */
FD3_API int fd3_energy_forces_stress(fd3_plan* plan, int64_t n_atoms, const double* d_pos_ang,
                             const int32_t* d_species, const double* h_cell_ang, const double* d_cell_ang,
                             double r_cut_ang, void* d_work, size_t work_bytes, double* d_energy,
                             double* d_forces, double* d_stress, void* stream);

/*
 * Direct pairwise D3(BJ) lattice sum in float64: the accuracy oracle of the reciprocal-space
 * methods (no reference counterpart; the reference checks its mesh methods against its own
 * Ewald path and torch-dftd, papercode/get_convergence.py). With the plan's smooth-cutoff CN and
 * low-rank C6 factors (C6_ij = sum_r lambda_r c_ir c_jr, core.py:323-386, 449-543) and the BJ
 * kernel of pair_pot.py:64:
 *   E = -1/2 sum'_{i,j,n} C6_ij [s6 / (r^6 + R0^6) + 3 s8 sqrt(Q_i Q_j) / (r^8 + R0^8)]
 * over every image pair closer than r_direct_ang (i = j at n = 0 excluded), plus the continuum
 * tail beyond r_direct; forces and stress analytic (pair terms, tail, CN chain). Same units and
 * output layout as fd3_energy_forces_stress; the plan's cnfunc must be FD3_CN_SMOOTH. Cost
 * grows as N r_direct^3: meant for accuracy checks, not for the timed path.
 */
FD3_API int fd3_direct_workspace_size(const fd3_plan* plan, int64_t n_atoms, const double* h_cell_ang,
                                      double r_cut_ang, double r_direct_ang, size_t* bytes);
FD3_API int fd3_direct_energy_forces_stress(fd3_plan* plan, int64_t n_atoms, const double* d_pos_ang,
                                            const int32_t* d_species, const double* h_cell_ang,
                                            const double* d_cell_ang, double r_cut_ang, double r_direct_ang,
                                            void* d_work, size_t work_bytes, double* d_energy,
                                            double* d_forces, double* d_stress, void* stream);

/*
 * Per-atom intermediates of the last compute call that used this workspace: the coordination
 * numbers after the optional cncorr correction (FourierD3.compute_cn_smooth, core.py:323-386)
 * and the rank-r C6 factors c[i, r] = sum_p w_ip V[Z_i, p, r] (core.py:449-478, 525-532),
 * row-major (n_atoms, r). n_atoms and n_bins must be those of that call (n_bins = 0 after
 * fd3_energy_edges). Either output may be NULL. Stream-ordered device-to-device copies.
 */
FD3_API int fd3_atom_terms(const fd3_plan* plan, int64_t n_atoms, int64_t n_bins, const void* d_work,
                           size_t work_bytes, double* d_cn, double* d_c6, void* stream);

/*
 * Neighbour list export (replaces matscipy.neighbours.neighbour_list("ijS"),
 * calculator.py:94-123): all directed pairs (i, j, S) with
 * |x_j - x_i + S.cell| < r_cut, both directions, self-images included, (i,i,0) excluded.
 * fd3_neighbor_count synchronises the stream and returns the pair count; fd3_neighbor_fill
 * writes rows sorted by i (within a row: cell-list order). h_capacity < count gives
 * FD3_ECAPACITY with the needed count in *h_count.
 */
FD3_API int fd3_neighbor_workspace_size(int64_t n_atoms, const double* h_cell_ang, double r_cut_ang, size_t* bytes);
FD3_API int fd3_neighbor_count(int64_t n_atoms, const double* d_pos_ang, const double* h_cell_ang, double r_cut_ang,
                       void* d_work, size_t work_bytes, int64_t* h_count, void* stream);
FD3_API int fd3_neighbor_fill(int64_t n_atoms, const double* d_pos_ang, const double* h_cell_ang, double r_cut_ang,
                      void* d_work, size_t work_bytes, int64_t capacity, int64_t* d_src, int64_t* d_dst,
                      int32_t* d_shift, int64_t* h_count, void* stream);

/*
 * Neighbour list with no allocation and no workspace argument. No counterpart in the
 * reference: it exists for callers that cannot allocate device memory themselves (an MD
 * engine or host runtime that owns all device memory and forbids raw allocations in its
 * timestep, or code with a fixed, pre-checked memory budget). Same inputs, outputs and
 * errors as fd3_neighbor_fill, but the cell-list scratch is a fixed 6 MiB device array
 * inside libfd3 (held on every GPU that loads the library until exit), enough for about
 * 65,000 atoms; larger inputs return FD3_EINVAL with the bytes needed. All calls share the
 * array and leave their data in it (the parts that must start at zero are cleared on each
 * call), so calls that overlap on the GPU race and must be serialised by the caller. The
 * first call on a device looks up the array's address with that device current; make it
 * before any stream capture. The address is cached for the life of the process, so the entry
 * point must not be used after cudaDeviceReset on that device.
 */
FD3_API int fd3_neighbor_fill_static(int64_t n_atoms, const double* d_pos_ang, const double* h_cell_ang,
                                     double r_cut_ang, int64_t capacity, int64_t* d_src, int64_t* d_dst,
                                     int32_t* d_shift, int64_t* h_count, void* stream);

/* Per-stage timing of the last call on this plan, from CUDA events recorded on the
 * launching stream between stages (cell_list, cn_c6, mesh_sort, spread, fft_r2c,
 * filter, fft_c2r, gather, cn_adjoint, finalize). fd3_profile_read waits for the last
 * event, writes milliseconds per stage and a comma-separated list of stage names. */
FD3_API int fd3_profile_enable(fd3_plan* plan, int32_t on);
FD3_API int fd3_profile_read(fd3_plan* plan, double* ms, int32_t max_stages, char* names, int32_t names_len,
                             int32_t* n_stages);

/* Last CUDA / cuFFT error text of the calling thread (static storage). */
FD3_API const char* fd3_last_error(void);
/* Number of kernel launches this library issued since load (for launch accounting). */
FD3_API int64_t fd3_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* FD3_H */
