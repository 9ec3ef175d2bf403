/*
 * tffb200.h -- C ABI of libtffb200.so, the sm_100a implementation of torchff's
 * fixed-charge nonbonded energy/force path (neighbour list, real-space Coulomb /
 * Lennard-Jones / Ewald pair terms, rank-0 PME).
 *
 * Conventions shared by every entry point
 *   - All array arguments are DEVICE pointers (the *_host functions excepted).
 *   - `dtype` selects the arithmetic: TFF_F32 = mixed precision (FP32 pair and spline
 *     arithmetic, 64-bit fixed-point force/grid accumulation, FP64 energies; results are
 *     bit-identical run to run), TFF_F64 = float64 throughout (FP64 atomics).
 *     Floating-point arrays are float* for TFF_F32 and double* for TFF_F64.
 *   - Coordinates are (N, 3) row-major; `box` is a (3, 3) row-major matrix whose rows
 *     are the box vectors (torchff/pbc.py), or NULL for an open system where allowed.
 *   - Index arrays are int64, pairs are (P, 2) row-major; a pair holding -1 is skipped.
 *   - Energies are written, gradients (dE/dx, dE/dq, ...) are written (not accumulated).
 *     A NULL gradient pointer skips that gradient.
 *   - Scratch memory is passed in by the caller as `workspace` of at least the size the
 *     matching *_workspace_bytes() reports; the library itself never calls cudaMalloc in
 *     these entry points (PME plans and system objects own their memory, see below).
 *   - Work is enqueued on `stream` (a cudaStream_t); nothing synchronises with the host
 *     except the *_host entry points. Calls of the entry points that take a workspace can
 *     be captured in a CUDA graph.
 *   - Return value: TFF_OK or an error code; tff_last_error() describes the last error
 *     of the calling thread.
 */
#ifndef TFFB200_H
#define TFFB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *tff_stream_t; /* identical to cudaStream_t */

enum tff_dtype { TFF_F32 = 0, TFF_F64 = 1 };

enum tff_status {
  TFF_OK = 0,
  TFF_ERR_INVALID = 1,     /* bad argument (shape, dtype, NULL, unsupported box) */
  TFF_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  TFF_ERR_CUFFT = 3,       /* a cuFFT call failed */
  TFF_ERR_WORKSPACE = 4,   /* workspace too small */
  TFF_ERR_CAPACITY = 5,    /* a fixed-capacity list overflowed (see tff_system_status) */
  TFF_ERR_TIMEOUT = 6      /* a wait on the server ran out of time */
};

int tff_version(void);
const char *tff_last_error(void);
/* Number of SMs the kernels size their grids for on the current device. */
int tff_device_sm_count(void);

/* ------------------------------------------------------------------------------
 * Neighbour lists
 * --------------------------------------------------------------------------- */

/* Replaces torch.ops.torchff.build_neighbor_list_nsquared / _out
 * (csrc/nblist/nblist_interface.cpp:5-6, csrc/nblist/nblist_nsquared_cuda.cu:129-199).
 * All pairs (i, j), i > j (i == j too when include_self), with |r_ij| <= cutoff under the
 * minimum image of `box` (NULL = open boundaries), skipping pairs listed in the symmetric
 * CSR exclusion structure (excl_row_ptr (N+1), excl_col; both NULL = none).
 * `pairs` (max_npairs, 2) is filled with -1 and the first min(found, max_npairs) rows
 * receive pairs; *npairs (device int32) receives the number FOUND, which may exceed
 * max_npairs (overflow). In TFF_F32 mode pairs within 1e-5 relative of the cutoff are
 * re-tested in FP64, so the pair set equals the FP64 one. Needs no workspace. */
int tff_nblist_nsquared(int dtype, int64_t natoms, const void *coords, const void *box,
                        double cutoff, const int64_t *excl_row_ptr, const int64_t *excl_col,
                        int include_self, int64_t *pairs, int64_t max_npairs, int32_t *npairs,
                        tff_stream_t stream);

/* Replaces torch.ops.torchff.build_neighbor_list_cell_list / _out
 * (csrc/nblist/nblist_interface.cpp:7-8, csrc/nblist/nblist_clist_cuda.cu:367-525).
 * Same output contract as tff_nblist_nsquared; needs a periodic `box` (any shape). Atoms
 * are binned on a Hilbert-ordered cell grid, grouped in 32-atom clusters and cluster pairs
 * are screened by bounding boxes (exact for orthorhombic boxes, conservative otherwise)
 * before a 32x32 warp tile test.
 * max_cluster_neighbors: capacity of each cluster's neighbour-cluster list (0 = default). */
size_t tff_nblist_cell_list_workspace_bytes(int dtype, int64_t natoms, int max_cluster_neighbors);
int tff_nblist_cell_list(int dtype, int64_t natoms, const void *coords, const void *box,
                         double cutoff, const int64_t *excl_row_ptr, const int64_t *excl_col,
                         int include_self, int64_t *pairs, int64_t max_npairs, int32_t *npairs,
                         int max_cluster_neighbors, void *workspace, size_t workspace_bytes,
                         tff_stream_t stream);

/* ------------------------------------------------------------------------------
 * Cluster-pair neighbour format
 * --------------------------------------------------------------------------- */

/* Replaces torch.ops.torchff.build_cluster_pairs (torchff/nblist.py:260-285,
 * csrc/nblist/nblist_cluster_pairs_cuda.cu:508-657). The format, all on the device:
 *   sorted_atoms  int32 (nclusters*32)    atom at each slot of the Hilbert-ordered 32-atom
 *                                         clusters, -1 after the last atom;
 *   tiles         int32 (2, tiles_cap)    cluster pairs (x, y), x <= y: every diagonal tile
 *                                         and every tile that holds an excluded pair; row 0 = x,
 *                                         row 1 = y, -1 padded;
 *   tile_masks    uint32 (tiles_cap, 32)  row (t, i): bit j set = pair (slot 32x+i, slot 32y+j)
 *                                         skipped (excluded, padding, or j <= i when x == y);
 *   entry_cluster int32 (entries_cap)     cluster x of each interacting entry, -1 padded;
 *   entry_atoms   int32 (entries_cap, 32) atoms of lower clusters that may interact with x
 *                                         (within the cutoff of x's bounding box), -1 padded.
 * Every atom pair within the cutoff and not excluded lies in exactly one tile or entry.
 * Exclusions: symmetric CSR (as for the neighbour lists), NULL = none.
 * counts (device int64 (3)) receives the numbers of tiles and entries NEEDED and a status
 * word (bit 0: a cluster has excluded partners in more than 64 clusters; bit 1: a cluster's
 * neighbour list overflowed max_cluster_neighbors); tiles / entries beyond the capacities
 * are not written. The outputs are filled with -1 first. nclusters = ceil(natoms / 32). */
size_t tff_cluster_pairs_workspace_bytes(int dtype, int64_t natoms, int max_cluster_neighbors);
int tff_cluster_pairs_build(int dtype, int64_t natoms, const void *coords, const void *box,
                            double cutoff, const int64_t *excl_row_ptr, const int64_t *excl_col,
                            int32_t *sorted_atoms, int32_t *tiles, uint32_t *tile_masks,
                            int64_t tiles_cap, int32_t *entry_cluster, int32_t *entry_atoms,
                            int64_t entries_cap, int64_t *counts, int max_cluster_neighbors,
                            void *workspace, size_t workspace_bytes, tff_stream_t stream);

/* Replaces torch.ops.torchff.decode_cluster_pairs (torchff/nblist.py:288-311,
 * csrc/nblist/nblist_cluster_pairs_cuda.cu:364-505, 659-716): every pair of the format within
 * the cutoff as int32 (larger, smaller) rows of `pairs` (max_npairs, 2), -1 filled first;
 * *npairs (device int32) = pairs FOUND (may exceed max_npairs). FP32 distances within 1e-5
 * relative of the cutoff are re-tested in FP64, so the pair set equals the FP64 one. */
int tff_cluster_pairs_decode(int dtype, int64_t natoms, const void *coords, const void *box,
                             double cutoff, const int32_t *sorted_atoms, int64_t nslots,
                             const int32_t *tiles, int64_t ntiles, const uint32_t *tile_masks,
                             const int32_t *entry_cluster, const int32_t *entry_atoms,
                             int64_t nentries, int32_t *pairs, int64_t max_npairs, int32_t *npairs,
                             tff_stream_t stream);

/* Replaces torch.ops.torchff.compute_nonbonded_energy_from_cluster_pairs (schema left
 * commented out at csrc/nonbonded/nonbonded_interface.cpp:7; kernel
 * csrc/nonbonded/nonbonded_cluster_pairs_cuda.cu): shifted (do_shift) or plain Coulomb + LJ
 * (Lorentz-Berthelot from per-atom sigma, epsilon) over the format, with the same pair math
 * as tff_nonbonded_atom_pairs. Outputs (each nullable): energy (1), its Coulomb part
 * energy_coulomb (1), dE/dx (N,3), dE/dsigma, dE/depsilon (0 where epsilon_i = 0), dE/dq. */
size_t tff_nonbonded_cluster_pairs_workspace_bytes(int dtype, int64_t natoms);
int tff_nonbonded_cluster_pairs(int dtype, int64_t natoms, const void *coords, const void *box,
                                const void *sigma, const void *epsilon, const void *charges,
                                double coul_constant, double cutoff, int do_shift,
                                const int32_t *sorted_atoms, int64_t nslots, const int32_t *tiles,
                                int64_t ntiles, const uint32_t *tile_masks,
                                const int32_t *entry_cluster, const int32_t *entry_atoms,
                                int64_t nentries, void *energy, void *energy_coulomb,
                                void *grad_coords, void *grad_sigma, void *grad_epsilon,
                                void *grad_charges, void *workspace, size_t workspace_bytes,
                                tff_stream_t stream);

/* Replaces torch.ops.torchff.compute_nonbonded_forces_from_cluster_pairs (schema left
 * commented out at csrc/nonbonded/nonbonded_interface.cpp:8): ADDS the shifted Coulomb + LJ
 * forces -dE/dx into `forces` (N,3). Workspace as tff_nonbonded_cluster_pairs. */
int tff_nonbonded_forces_cluster_pairs(int dtype, int64_t natoms, const void *coords,
                                       const void *box, const void *sigma, const void *epsilon,
                                       const void *charges, double coul_constant, double cutoff,
                                       const int32_t *sorted_atoms, int64_t nslots,
                                       const int32_t *tiles, int64_t ntiles,
                                       const uint32_t *tile_masks, const int32_t *entry_cluster,
                                       const int32_t *entry_atoms, int64_t nentries, void *forces,
                                       void *workspace, size_t workspace_bytes, tff_stream_t stream);

/* ------------------------------------------------------------------------------
 * Pair terms over an explicit pair list
 * --------------------------------------------------------------------------- */

/* Workspace of every *_atom_pairs entry point; ntypes = size of the LJ type table
 * (0 when type tables are not used). */
size_t tff_pairs_workspace_bytes(int dtype, int64_t natoms, int64_t ntypes);

/* Replaces torch.ops.torchff.compute_nonbonded_energy_from_atom_pairs
 * (csrc/nonbonded/nonbonded_interface.cpp:9, csrc/nonbonded/nonbonded_atom_pairs_cuda.cu:17-141, 144-238).
 * E = sum_{r<=rc} k q_i q_j (1/r - [do_shift]/rc) + 4 eps_ij ((s_ij/r)^12 - (s_ij/r)^6),
 * s_ij = (s_i+s_j)/2, eps_ij = sqrt(eps_i eps_j). Gradients: dE/dx (N,3), dE/dsigma (N),
 * dE/depsilon (N; pairs with eps_ij = 0 contribute 0), dE/dq (N). */
int tff_nonbonded_atom_pairs(int dtype, int64_t natoms, const void *coords, int64_t npairs,
                             const int64_t *pairs, const void *box, const void *sigma,
                             const void *epsilon, const void *charges, double coul_constant,
                             double cutoff, int do_shift, void *energy, void *grad_coords,
                             void *grad_sigma, void *grad_epsilon, void *grad_charges,
                             void *workspace, size_t workspace_bytes, tff_stream_t stream);

/* No counterpart in the reference. tff_nonbonded_atom_pairs without a workspace, for
 * callers that cannot allocate device memory: a force plugin inside a molecular-dynamics
 * engine that owns every device allocation and gives the plugin only its input and output
 * buffers, or a time-critical loop that must never reach an allocator (an allocation can
 * synchronise the device or fail mid-run). This entry point calls no cudaMalloc/cudaFree
 * and no allocating library routine; its scratch is a static device array inside
 * libtffb200 (about 3 MiB, held by every GPU that loads the library until exit), so natoms
 * is limited to TFF_NOALLOC_MAX_ATOMS (larger inputs return TFF_ERR_INVALID). The first
 * call on each device (and the first after a device reset) looks the array up with
 * cudaGetSymbolAddress: make it before any stream capture. All calls share the array
 * (cleared at the start of each call, it keeps the last call's contents): calls that
 * overlap on the GPU race, so serialise them. Inputs, outputs and results are those of
 * tff_nonbonded_atom_pairs. */
#define TFF_NOALLOC_MAX_ATOMS 65536
int tff_nonbonded_atom_pairs_noalloc(int dtype, int64_t natoms, const void *coords,
                                     int64_t npairs, const int64_t *pairs, const void *box,
                                     const void *sigma, const void *epsilon, const void *charges,
                                     double coul_constant, double cutoff, int do_shift,
                                     void *energy, void *grad_coords, void *grad_sigma,
                                     void *grad_epsilon, void *grad_charges, tff_stream_t stream);

/* Replaces torch.ops.torchff.compute_nonbonded_forces_from_atom_pairs
 * (csrc/nonbonded/nonbonded_interface.cpp:10, csrc/nonbonded/nonbonded_atom_pairs_cuda.cu:263-305):
 * ADDS the shifted Coulomb + LJ forces -dE/dx into `forces` (N,3). */
int tff_nonbonded_forces_atom_pairs(int dtype, int64_t natoms, const void *coords,
                                    int64_t npairs, const int64_t *pairs, const void *box,
                                    const void *sigma, const void *epsilon, const void *charges,
                                    double coul_constant, double cutoff, void *forces,
                                    void *workspace, size_t workspace_bytes, tff_stream_t stream);

/* Replaces torch.ops.torchff.compute_coulomb_energy
 * (csrc/coulomb/coulomb_interface.cpp:5, csrc/coulomb/coulomb_cuda.cu:17-204).
 * Gradients dE/dx and dE/dq (dE/dq_i = sum_j k q_j (1/r - [do_shift]/rc), no division by q_i). */
int tff_coulomb_atom_pairs(int dtype, int64_t natoms, const void *coords, int64_t npairs,
                           const int64_t *pairs, const void *box, const void *charges,
                           double coul_constant, double cutoff, int do_shift, void *energy,
                           void *grad_coords, void *grad_charges, void *workspace,
                           size_t workspace_bytes, tff_stream_t stream);

/* Replaces torch.ops.torchff.compute_lennard_jones_energy
 * (csrc/vdw/vdw_interface.cpp:6, csrc/vdw/vdw.cu:83-344).
 * atom_types == NULL: sigma/epsilon are per pair (P,), gradients per pair.
 * atom_types != NULL: sigma/epsilon are (ntypes, ntypes) tables, gradients are tables. */
int tff_lennard_jones_atom_pairs(int dtype, int64_t natoms, const void *coords, int64_t npairs,
                                 const int64_t *pairs, const void *box, const void *sigma,
                                 const void *epsilon, double cutoff, const int64_t *atom_types,
                                 int64_t ntypes, void *energy, void *grad_coords,
                                 void *grad_sigma, void *grad_epsilon, void *workspace,
                                 size_t workspace_bytes, tff_stream_t stream);

/* Replaces torch.ops.torchff.compute_multipolar_energy_from_atom_pairs at rank 0
 * (csrc/multipoles/multipoles_interface.cpp:6, csrc/multipoles/multipoles.cu:24-152,
 * csrc/multipoles/multipoles_forward.cuh:356-617).
 * E = prefactor [sum_{pairs, r<=rc} q_i q_j D(r)/r + sum_{excl, r<=rc} q_i q_j (D(r)-1)/r]
 * with D = erfc(ewald_alpha r) when ewald_alpha >= 0, else D = 1 and no exclusion term.
 * Gradients dE/dx and dE/dq. */
int tff_ewald_real_atom_pairs(int dtype, int64_t natoms, const void *coords, const void *box,
                              int64_t npairs, const int64_t *pairs, int64_t npairs_excl,
                              const int64_t *pairs_excl, const void *charges, double cutoff,
                              double ewald_alpha, double prefactor, void *energy,
                              void *grad_coords, void *grad_charges, void *workspace,
                              size_t workspace_bytes, tff_stream_t stream);

/* ------------------------------------------------------------------------------
 * Bonded terms (flexible water): harmonic bonds and angles
 * --------------------------------------------------------------------------- */

/* Workspace of every bonded entry point below (nterms = bonds or angles of the call). */
size_t tff_bonded_workspace_bytes(int dtype, int64_t natoms, int64_t nterms);

/* Replaces torch.ops.torchff.compute_harmonic_bond_energy (csrc/bond/bond_interface.cpp:5,
 * csrc/bond/harmonic_bond_cuda.cu:78-142; torchff/bond.py:9-43):
 * E = sum 1/2 k_m (r_m - b0_m)^2, r_m = |x_j - x_i| for bonds (M,2) int64 (no periodic image,
 * as the reference). Outputs (each nullable): energy (1), dE/dx (N,3), dE/db0 (M,), dE/dk (M,). */
int tff_harmonic_bond(int dtype, int64_t natoms, const void *coords, int64_t nbonds,
                      const int64_t *bonds, const void *b0, const void *k, void *energy,
                      void *grad_coords, void *grad_b0, void *grad_k, void *workspace,
                      size_t workspace_bytes, tff_stream_t stream);

/* Replaces torch.ops.torchff.compute_harmonic_bond_forces (csrc/bond/bond_interface.cpp:6,
 * csrc/bond/harmonic_bond_cuda.cu:145-175): ADDS -dE/dx into `forces` (N,3). */
int tff_harmonic_bond_forces(int dtype, int64_t natoms, const void *coords, int64_t nbonds,
                             const int64_t *bonds, const void *b0, const void *k, void *forces,
                             void *workspace, size_t workspace_bytes, tff_stream_t stream);

/* Replaces torch.ops.torchff.compute_harmonic_angle_energy (csrc/angle/angle_interface.cpp:5,
 * csrc/angle/harmonic_angle_cuda.cu:104-169; torchff/angle.py:78-112): E = sum 1/2 k (theta -
 * theta0)^2, theta the angle at the central atom j of each (i, j, k) row of angles (M,3) int64.
 * Outputs (each nullable): energy (1), dE/dx (N,3), dE/dtheta0 (M,), dE/dk (M,). Straight angles
 * use sin(theta) >= 1e-15 instead of the unbounded derivative. */
int tff_harmonic_angle(int dtype, int64_t natoms, const void *coords, int64_t nangles,
                       const int64_t *angles, const void *theta0, const void *k, void *energy,
                       void *grad_coords, void *grad_theta0, void *grad_k, void *workspace,
                       size_t workspace_bytes, tff_stream_t stream);

/* Replaces torch.ops.torchff.compute_harmonic_angle_forces (csrc/angle/angle_interface.cpp:6,
 * csrc/angle/harmonic_angle_cuda.cu:172-204): ADDS -dE/dx into `forces` (N,3). */
int tff_harmonic_angle_forces(int dtype, int64_t natoms, const void *coords, int64_t nangles,
                              const int64_t *angles, const void *theta0, const void *k,
                              void *forces, void *workspace, size_t workspace_bytes,
                              tff_stream_t stream);

/* Replaces torch.ops.torchff.compute_angles and its backward (csrc/angle/angle_interface.cpp:7,
 * csrc/angle/angles_cuda.cu:83-160; torchff/angle.py:8-55): theta (M,) of every angle (nullable);
 * with grad_theta (M,) also dE/dx = sum grad_theta dtheta/dx into grad_coords (N,3). */
int tff_angles(int dtype, int64_t natoms, const void *coords, int64_t nangles,
               const int64_t *angles, void *theta, const void *grad_theta, void *grad_coords,
               void *workspace, size_t workspace_bytes, tff_stream_t stream);

/* ------------------------------------------------------------------------------
 * PME reciprocal space (rank 0, order-6 B-splines, cubic K x K x K grid)
 * --------------------------------------------------------------------------- */

typedef struct tff_pme_plan_s *tff_pme_plan;

/* Creates the cuFFT R2C/C2R plans (cuFFT allocates its own work area here). */
int tff_pme_plan_create(int dtype, int K, tff_pme_plan *plan);
int tff_pme_plan_destroy(tff_pme_plan plan);
size_t tff_pme_workspace_bytes(tff_pme_plan plan, int64_t natoms);

/* Replaces torch.ops.torchff.pme_long_range at rank 0 (csrc/pme/pme_interface.cpp:6-9,
 * csrc/pme/pme.cu:19-246): forward (spread, rFFT, influence function, irFFT, self term)
 * AND the gather the reference runs in backward, in one call.
 * Outputs: energy (scalar) = 1/2 sum q phi - (alpha/sqrt(pi)) sum q^2 in e^2/nm units;
 * phi (N) = dE/dq (self term included); grad_coords (N,3) = dE/dx. Any output may be NULL
 * except energy. moduli: the B-spline moduli (K), (K), (K/2+1) as torchff/bsplines.py
 * computes them (same dtype as coords). */
int tff_pme_long_range(tff_pme_plan plan, int64_t natoms, const void *coords, const void *box,
                       const void *charges, double alpha, const void *xmoduli,
                       const void *ymoduli, const void *zmoduli, void *energy, void *phi,
                       void *grad_coords, void *workspace, size_t workspace_bytes,
                       tff_stream_t stream);

/* ------------------------------------------------------------------------------
 * Fused fixed-charge system: cluster-pair neighbour build + fused real-space
 * LJ / erfc-Coulomb with exclusion correction + PME, energy and forces in one call.
 * This is the evaluation of examples/tip3p/model.py:100-133 (nonbonded terms, plus the
 * harmonic bonds and angles of a flexible model through tff_system_set_bonded).
 * --------------------------------------------------------------------------- */

typedef struct tff_system_s *tff_system;

typedef struct tff_system_desc {
  int dtype;                  /* TFF_F32 (mixed) or TFF_F64 */
  int64_t natoms;
  double cutoff;              /* nm */
  double ewald_alpha;         /* nm^-1 */
  int pme_grid;               /* K (cubic grid), 0 disables reciprocal space */
  double coul_constant;       /* 138.935456 kJ mol^-1 nm e^-2 */
  int max_cluster_neighbors;  /* 0 = default */
} tff_system_desc;

/* Creates a system, copying per-atom parameters from HOST arrays (float64):
 * charges (N), sigma (N), epsilon (N) (Lorentz-Berthelot combining) and the exclusion
 * pairs (nexcl, 2) int64 (both orders implied; self pairs ignored). Excluded pairs get no
 * LJ and the Ewald exclusion correction -k q_i q_j erf(alpha r)/r. Owns device memory. */
int tff_system_create(const tff_system_desc *desc, const double *charges, const double *sigma,
                      const double *epsilon, int64_t nexcl, const int64_t *excl_pairs,
                      tff_system *sys);
int tff_system_destroy(tff_system sys);
/* Overwrites per-atom parameters (device arrays of the system dtype, may be NULL to keep). */
int tff_system_set_parameters(tff_system sys, const void *charges, const void *sigma,
                              const void *epsilon, tff_stream_t stream);
/* Adds (or, with nbonds = nangles = 0, removes) the harmonic bonds and angles of a flexible
 * model (examples/tip3p/model.py:105-106: HarmonicBond + HarmonicAngle, torchff/bond.py,
 * torchff/angle.py) to the system. HOST arrays: bonds (nbonds, 2) int64, b0, kb (nbonds);
 * angles (nangles, 3) int64 (central atom in the middle), theta0 (rad), ktheta (nangles).
 * They are evaluated in every tff_system_eval / _eval_host / _eval_grads (energy and forces;
 * bond lengths use no periodic image, as the reference); tff_system_hvp then returns
 * TFF_ERR_INVALID. Synchronises the device; call it outside stream capture. */
int tff_system_set_bonded(tff_system sys, int64_t nbonds, const int64_t *bonds, const double *b0,
                          const double *kb, int64_t nangles, const int64_t *angles,
                          const double *theta0, const double *ktheta);
/* Evaluates energy and forces with device-resident inputs. coords (N,3), box (3,3) in the
 * system dtype; energy (device double, 1) total in kJ/mol; forces (N,3) system dtype,
 * = -dE/dx; grad_charges (N) optional dE/dq. energy_terms (device double) optional:
 * real-space pairs, exclusion correction, reciprocal, self (4 values), then bonds and
 * angles (6 values) when the system has bonded terms. */
int tff_system_eval(tff_system sys, const void *coords, const void *box, double *energy,
                    void *forces, void *grad_charges, double *energy_terms, tff_stream_t stream);
/* Same with HOST buffers: copies coords/box in, evaluates, copies energy/forces out and
 * synchronises `stream`. coords/box/forces are float64 host arrays whatever the dtype.
 * When coords and forces are page-locked (cudaHostAlloc / cudaHostRegister) the copies and
 * the evaluation are one CUDA-graph launch, kept for the last (coords, forces) pair seen and
 * captured again when either pointer changes. Returns TFF_ERR_CAPACITY when a cluster's
 * neighbour list overflowed its capacity (max_cluster_neighbors): the energy and forces it
 * wrote then miss pairs. */
int tff_system_eval_host(tff_system sys, const double *coords, const double *box,
                         double *energy, double *forces, tff_stream_t stream);
/* Device status word of the last evaluation (bit 0: a cluster neighbour list overflowed,
 * bit 1: fixed-point accumulator overflow guard tripped). Synchronises `stream`. */
int tff_system_status(tff_system sys, tff_stream_t stream, int *status);

/* Stage timing. A timer holds TFF_TIMER_EVENTS CUDA events; tff_system_eval_timed records
 * them at the stage boundaries of one evaluation (also inside a CUDA-graph capture, as
 * event-record nodes): 0 start, 1 cluster build done, 2 real-space tile kernel done,
 * 3 PME spread + FFTs + influence function done, 4 PME gather done, 5 finalize done.
 * tff_timer_elapsed_ms waits for event `to` and returns the time between two events. */
#define TFF_TIMER_EVENTS 6
typedef struct tff_timer_s *tff_timer;
int tff_timer_create(tff_timer *timer);
int tff_timer_destroy(tff_timer timer);
int tff_timer_elapsed_ms(tff_timer timer, int from, int to, float *ms);
int tff_system_eval_timed(tff_system sys, const void *coords, const void *box, double *energy,
                          void *forces, tff_timer timer, tff_stream_t stream);
/* First derivatives with respect to the per-atom parameters too (energy, forces = -dE/dx,
 * dE/dq, dE/dsigma, dE/depsilon; any output may be NULL). Epsilon enters the LB mean as
 * sqrt(eps_i eps_j); dE/deps_i is reported as 0 where eps_i = 0 (the derivative of sqrt is
 * unbounded there). The reference's pair op divides by eps_ij instead
 * (csrc/nonbonded/nonbonded_atom_pairs_cuda.cu:126-129). */
int tff_system_eval_grads(tff_system sys, const void *coords, const void *box, double *energy, void *forces,
                          void *grad_charges, void *grad_sigma, void *grad_epsilon, tff_stream_t stream);
/* Second derivatives for force matching (no reference counterpart: the reference has no
 * double backward on CUDA). For a coordinate direction u (N, 3) writes the derivatives of
 * s(x, q, sigma, eps) = sum_i u_i . dE/dx_i with respect to the coordinates (N, 3), charges,
 * sigma and epsilon (N each; NULL skips). One call rebuilds the cluster lists and evaluates
 * the real-space and PME second derivatives (the PME part spreads the directional grid
 * P = sum_i q_i u_i . grad theta_i and convolves it like the charge grid). */
int tff_system_hvp(tff_system sys, const void *coords, const void *box, const void *direction, void *hvp_coords,
                   void *hvp_charges, void *hvp_sigma, void *hvp_epsilon, tff_stream_t stream);
/* Number of kernels of this library one tff_system_eval launches (cuFFT's excluded). */
int tff_system_kernel_launches(tff_system sys);

/* ------------------------------------------------------------------------------
 * Batches: many independent periodic systems per evaluation (serving)
 *
 * No reference counterpart: the reference evaluates one system per call (its torch-sim
 * wrapper, examples/tip3p/md_torchsim.py:113-140, rejects n_systems != 1). A batch object
 * owns device memory for up to max_systems systems holding max_atoms atoms and
 * max_grid_points PME grid points (sum of K^3) in total; every stage of an evaluation is
 * one launch over all systems (each with its own box, cell grid and PME grid K), and each
 * system's result is the one a single-system evaluation of the same dtype gives (mixed
 * precision: bit-identical whatever else is in the batch). Same physics as tff_system_*;
 * cutoff, Ewald alpha and the Coulomb constant are shared by the batch.
 * Per system: 1 <= natoms <= 16384, 6 <= K <= 96 (TFF_F32) or 64 (TFF_F64). The
 * reciprocal-space transforms of a batch are a direct 3-D DFT of every grid (one launch per
 * axis pass for all sizes), not cuFFT; results match the single-system (cuFFT) path to FP
 * rounding.
 * --------------------------------------------------------------------------- */
typedef struct tff_batch_s *tff_batch;

typedef struct tff_batch_desc {
  int dtype;
  int max_systems;
  int64_t max_atoms;
  int64_t max_grid_points;
  double cutoff;
  double ewald_alpha;
  double coul_constant;
  int max_cluster_neighbors;  /* 0 = 512, enough for any accepted system */
  double atoms_per_cell;      /* cell grid occupancy target, 0 = 8 */
} tff_batch_desc;

/* Device bytes a batch with this description allocates (for admission planning). */
size_t tff_batch_device_bytes(const tff_batch_desc *desc);
int tff_batch_create(const tff_batch_desc *desc, tff_batch *batch);
int tff_batch_destroy(tff_batch batch);
/* natoms[nsys], pme_grid[nsys]: HOST arrays. Device arrays, systems one after another in
 * caller order: coords (sum natoms, 3), boxes (nsys, 3, 3), charges / sigma / epsilon
 * (sum natoms), excl (sum natoms, 8) int32 excluded partners as atom indices within
 * their own system, -1 padded; out: energies (nsys) float64, forces (sum natoms, 3) in the batch dtype.
 * The host part (system table, work-unit offsets) runs in the call; the call returns once
 * the work is enqueued. One evaluation at a time per batch object and stream.
 * Every launch shape of the device part depends on the batch's capacity and the DFT size
 * class (grid sides up to 52, or larger) alone; the composition is uploaded with the
 * system table. So when a call repeats the previous call's device pointers and DFT class,
 * the device part is captured in a CUDA graph, and later calls with those pointers and
 * that class replay it whatever systems they hold (up to 8 graphs per batch object). */
int tff_batch_eval(tff_batch batch, int nsys, const int64_t *natoms, const int *pme_grid, const void *coords,
                   const void *boxes, const void *charges, const void *sigma, const void *epsilon,
                   const int *excl, double *energies, void *forces, tff_stream_t stream);
int tff_batch_status(tff_batch batch, tff_stream_t stream, int *status);
int tff_batch_kernel_launches(tff_batch batch);
/* No counterpart in the reference. Evaluations of this batch object so far that ran as a
 * replay of a captured graph. */
int64_t tff_batch_graph_launches(tff_batch batch);

/* ------------------------------------------------------------------------------
 * Server: continuous batching of requests over tff_batch (no reference counterpart)
 *
 * A worker thread keeps `lanes` batches in flight, each on its own stream with its own
 * device memory (hbm_budget_bytes split evenly; a lane's capacity in atoms and PME grid
 * points is the largest that fits its share). Whenever a lane is free and requests are
 * queued, it takes as many as fit (in submission order) and evaluates them as one batch,
 * so requests arriving while other batches run start as soon as a lane frees up, and
 * the lanes' batches overlap on the device. Inputs are copied at submission; energy and
 * forces (float64) are written to the request's host buffers when it completes.
 * --------------------------------------------------------------------------- */
typedef struct tff_server_s *tff_server;

typedef struct tff_server_desc {
  int dtype;
  int lanes;                    /* batches in flight, 1..16 */
  int max_systems_per_batch;
  size_t hbm_budget_bytes;      /* device memory of all lanes together */
  double grid_points_per_atom;  /* lane PME grid capacity per atom of capacity (water at 0.1 nm: ~12) */
  double cutoff;
  double ewald_alpha;
  double coul_constant;
  double atoms_per_cell;        /* cell grid occupancy target, 0 = 8 */
} tff_server_desc;

typedef struct tff_request {
  int64_t natoms;               /* 1..16384 */
  int pme_grid;                 /* K, 6..96 (TFF_F32) or 6..64 (TFF_F64) */
  const double *coords;         /* host (natoms, 3) */
  const double *box;            /* host (3, 3), rows are box vectors */
  const double *charges;        /* host (natoms) */
  const double *sigma;          /* host (natoms) */
  const double *epsilon;        /* host (natoms) */
  int64_t nexcl;                /* excluded pairs (i, j), system-local indices */
  const int64_t *excl_pairs;    /* host (nexcl, 2) */
  double *energy;               /* host out, written on completion */
  double *forces;               /* host out (natoms, 3), written on completion */
} tff_request;

typedef struct tff_server_stats {
  int64_t submitted, systems_launched, systems_done, batches;
  int64_t max_batch_systems, max_batch_atoms, max_lanes_in_flight;
  int64_t lane_max_atoms, lane_max_grid_points, lane_device_bytes;
  double now;                   /* seconds since the server was created (the request clock) */
} tff_server_stats;

int tff_server_create(const tff_server_desc *desc, tff_server *server);
/* Finishes the queued requests, then stops the worker and frees everything. */
int tff_server_destroy(tff_server server);
int tff_server_submit(tff_server server, const tff_request *request, int64_t *ticket);
/* Blocks until the request is done (timeout_s < 0: no limit); returns its status. */
int tff_server_wait(tff_server server, int64_t ticket, double timeout_s);
int tff_server_poll(tff_server server, int64_t ticket, int *done);
/* Submission, batch start and completion times of a request on the server clock. */
int tff_server_request_times(tff_server server, int64_t ticket, double *t_submit, double *t_start,
                             double *t_done);
/* Forgets a finished request; refused (TFF_ERR_INVALID) while another thread is inside
 * tff_server_wait on it. */
int tff_server_release(tff_server server, int64_t ticket);
/* Blocks until every submitted request is done. */
int tff_server_drain(tff_server server, double timeout_s);
int tff_server_get_stats(tff_server server, tff_server_stats *stats);
/* hold != 0: no new batch starts (submissions keep queueing); hold == 0 resumes. */
int tff_server_hold(tff_server server, int hold);

#ifdef __cplusplus
}
#endif

#endif /* TFFB200_H */
