/*
 * sirocco_solve.h -- C ABI of the B200 batched dense-solve engine.
 *
 * Part 1 is a link-compatible drop-in for the reference's linear-algebra layer:
 * the same prototypes, row-major double layout, size argument and return codes
 * as the reference's GSL build (source/templates.h:358-360, implemented in
 * source/matrix_cpu.c) plus the lifecycle names of its optional CUDA build
 * (source/matrix_gpu.h:16-24).  Part 2 adds batched entry points that take a
 * whole cycle's systems in one call.
 *
 * Return codes (the reference's GSL build, source/matrix_cpu.c):
 *   solve : 0 ok; 4 singular (an exact zero on the diagonal of U, lu.c:540);
 *           2 / 3 the first row failing the relative / absolute residual check
 *           (matrix_cpu.c:162-187), x still written.
 *   invert: 0 ok; 1 singular (GSL_EDOM); 8 out of memory (GSL_ENOMEM).
 * The FP64 kernels reproduce GSL's factorisation bit for bit, so the codes match
 * the reference's exactly; the mixed-precision mode re-runs any system whose
 * code could differ in exact FP64.
 */
#ifndef SIROCCO_SOLVE_H
#define SIROCCO_SOLVE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- part 1 -- */

/* Replaces solve_matrix (source/matrix_cpu.c:310, prototype templates.h:359).
   Solves A x = b for one n x n row-major system in host memory.  a_matrix is
   read only (the reference factorises it in place; callers free it right
   after).  x_matrix is written unless the code is 4.  nplasma is only used in
   messages, as in the reference. */
int solve_matrix(double *a_matrix, double *b_matrix, int size, double *x_matrix, int nplasma);

/* Replaces invert_matrix (source/matrix_cpu.c:338, prototype templates.h:360).
   inverted_matrix is written only when the return code is 0. */
int invert_matrix(double *matrix, double *inverted_matrix, int num_rows);

/* Replaces get_matrix_error_string (source/matrix_cpu.c:274): the text of a
   solve_matrix code, as the reference's GSL build words it. */
const char *get_matrix_error_string(int error_code);

/* Replace the lifecycle hooks of the reference's CUDA build
   (source/matrix_gpu.cu:125 cusolver_create, :159 cusolver_destroy, :50
   cusolver_get_error_string).  create is idempotent and binds the calling
   thread to the current CUDA device; destroy is a no-op when nothing was
   created.  Both return 0 on success, else a CUDA error code. */
int cusolver_create(void);
int cusolver_destroy(void);
const char *cusolver_get_error_string(int error);

/* Aliases of solve_matrix / invert_matrix under the names of the reference's
   CUDA build (source/matrix_gpu.cu:264, :332; matrix_gpu.h:20-21). */
int gpu_solve_matrix(double *a_matrix, double *b_vector, int size, double *x_vector);
int gpu_invert_matrix(double *matrix, double *inverse, int num_rows);

/* ---------------------------------------------------------------- part 2 -- */

/* Precision modes of the batched entry points. */
#define SIROCCO_FP64 0   /* GSL-exact FP64 factorisation                         */
#define SIROCCO_MIXED 1  /* equilibrated FP32 factorisation + FP64 refinement,
                            exact FP64 for any system whose result or code the
                            refinement cannot vouch for                          */
#define SIROCCO_FAST 2   /* inverses of certified matrices -- nonsingular
                            M-matrices: diagonal entries within [1/4, 4],
                            off-diagonal entries <= 0, every row strictly
                            dominant by a relative margin of at least 1e-5,
                            as the macro-atom jumping
                            matrix N = I - Q/Q_norm is wherever every level can
                            deactivate -- by FP64 Gauss-Jordan without pivoting
                            (code 0, as GSL's, and within ~1e-11 of GSL's
                            inverse); every other system, and every solve, by
                            the GSL-exact FP64 path of SIROCCO_FP64             */

/* Library error codes returned by the batched entry points (per-system codes
   go to status[]); positive values are CUDA error codes. */
#define SIROCCO_OK 0
#define SIROCCO_EINVAL (-1)   /* bad argument: nsys < 0, n < 1, null pointer   */
#define SIROCCO_ESIZE (-2)    /* a system larger than the engine supports      */
#define SIROCCO_EMODE (-3)    /* unknown precision mode                        */
#define SIROCCO_MAX_N 1024  /* shared-memory bound of the n > 256 path */

/* Batched solve, called once per ionisation cycle (or once per n_e round of
   the lock-step ion iteration) over all cells' systems.  The layout arrays
   n[nsys], offA[nsys] (element offset of each matrix in A) and offv[nsys]
   (element offset of each right-hand side in b and solution in x) are HOST
   arrays; A, b, x and status may all be host or all be device pointers.
   Returns 0, a negative library code, or a CUDA error code; status[s] holds the
   reference code of system s.  For a singular system x is left unspecified. */
int solve_matrix_batched(int nsys, const int *n, const int64_t *offA, const double *A,
                         const int64_t *offv, const double *b, double *x, int *status);

/* Batched inverse, called once per cycle from the matom-matrix cell loop.
   status[s] is invert_matrix's code: 0, 1 (an exact zero pivot in GSL's LU) or
   21 (GSL_ESING: an infinite pivot, which LU_invx turns into a zero on the
   diagonal of U^-1), the output left untouched for 1 and 21.  In SIROCCO_FAST
   mode a system may also get -3: the certified kernel's staging copy did not
   arrive within its bounded wait (about a second), so the system was not
   processed; no correct run produces it. */
int invert_matrix_batched(int nsys, const int *n, const int64_t *offA, const double *A,
                          double *Ainv, int *status);

/* Precision mode used by the two batched calls above (default SIROCCO_FP64). */
int sirocco_set_precision(int mode);

/* Plans: the size bucketing of one batch layout, its device-side copy and a
   captured launch sequence, reusable every cycle.  kind 0 = solve, 1 = invert.
   Layout arrays are host arrays (offv ignored for kind 1). */
typedef struct sirocco_plan sirocco_plan;
int sirocco_plan_create(sirocco_plan **plan, int kind, int nsys, const int *n, const int64_t *offA,
                        const int64_t *offv, int mode);
/* Enqueue the whole batch on `stream` (a cudaStream_t, 0 = legacy default).
   All pointers are device pointers; b is ignored for an inverse; diag may be
   null (bits 0-7: refinement iterations; bit 8: the result came from the
   GSL-exact FP64 path, always so in FP64 mode; bit 9: refinement stalled;
   bit 10: condition estimate above the mixed-mode limit). */
int sirocco_plan_execute(sirocco_plan *plan, const double *A, const double *b, double *out,
                         int *status, int *diag, void *stream);
/* Number of kernel launches one execute issues. */
int sirocco_plan_launches(const sirocco_plan *plan);
int sirocco_plan_destroy(sirocco_plan *plan);

/* Text of the last library error on this thread. */
const char *sirocco_last_error(void);

/* Lock-step ionisation balance: the n_e iteration of matrix_ion_populations
   (source/matrix_ion.c:219-382) for ncell cells at once, one batched solve per
   round over every unfinished cell.  Ions 0..nions-1 form nelem elements;
   element e holds ions elem_first[e] .. elem_first[e]+elem_n[e]-1 and istate[]
   is each ion's charge + 1 (ion[].istate).  h_elem is hydrogen's element (-1:
   none).  elem_dens[c*nelem + e] is the element number density of cell c.
   ne[c] (in: the starting n_e, out: the converged one) and den[c*nions + i]
   (in: starting ion fractions of each element, out: converged ones) are
   updated only for cells that converge.  Each round the library calls
   `assemble` for the cells still iterating: for cell cells[i] at n_e ne[i] and
   neutral / ionised hydrogen densities nh1[i], nh2[i] it fills the rate matrix
   (populate_ion_rate_matrix, matrix_ion.c:445-659) as one row-major block per
   element, cell after cell (A) and the matching right-hand sides (b, nions per
   cell); a nonzero return aborts with SIROCCO_EINVAL.  After each solve the
   cell follows the reference: populations floored at DENSITY_MIN (1e-20), new
   n_e from the ion charges, converged when |n_e - n_e'| / n_e' < 0.03 or
   n_e' < 1e-6, otherwise n_e <- (n_e + n_e') / 2, at most 200 rounds.
   status[c]: 0 converged, -1 a singular block (solve_matrix code 4, the
   reference's return -1), -2 no convergence in 200 rounds.  iters[c]: rounds
   used.  The solves use the precision mode of sirocco_set_precision.  All
   arrays are host arrays. */
typedef int (*sirocco_ion_assemble_fn)(void *user, int ncell, const int *cells, const double *ne, const double *nh1,
                                       const double *nh2, double *A, double *b);
int ion_populations_lockstep(int ncell, int nions, int nelem, const int *elem_first, const int *elem_n,
                             const int *istate, int h_elem, const double *elem_dens, double *ne, double *den,
                             sirocco_ion_assemble_fn assemble, void *user, int *status, int *iters);

/* The atomic data populate_ion_rate_matrix (source/matrix_ion.c:444-659) reads:
   the ele[] / ion[] fields it tests, the inner-shell rates with their electron
   yields (inner_cross[], inner_elec_yield[]) and the charge-exchange entries
   (charge_exchange[]).  Element e owns ions elem_first[e] .. elem_first[e] +
   elem_n[e] - 1 in stage order (stage 1 = neutral).  Host arrays. */
typedef struct sirocco_ion_table {
  int nions, nelem;
  const int *elem_z;            /* [nelem] atomic number */
  const int *elem_first;        /* [nelem] first ion */
  const int *elem_n;            /* [nelem] ions of the element */
  const int *elem_istate_max;   /* [nelem] highest stage */
  const int *ion_istate;        /* [nions] stage */
  const int *ion_di;            /* [nions] dere_di_flag */
  const int *ion_dr;            /* [nions] drflag */
  int n_inner;
  const int *inner_nion;        /* [n_inner] ion depopulated by inner-shell rate m */
  const int *inner_yield;       /* [n_inner] its row of yield_prob, -1 without yield data */
  int n_yield;
  const double *yield_prob;     /* [n_yield][10] probability of 1..10 ejected electrons */
  int ncx;
  const int *cx_nion1;          /* [ncx] ion ionised by charge exchange */
  const int *cx_nion2;          /* [ncx] its partner; entries count when that is hydrogen */
} sirocco_ion_table;

/* Per-cell coefficients, cell after cell: pi, rr (pi_rates, rr_rates), di, qr,
   dr (di_coeffs, qrecomb_coeffs, dr_coeffs) and cxr
   (charge_exchange_recomb_rates), nions each; cxi
   (charge_exchange_ioniz_rates), ncx each; inner (inner_rates), n_inner each.
   Host arrays. */
typedef struct sirocco_ion_rates {
  const double *pi, *rr, *di, *qr, *dr, *cxr, *cxi, *inner;
} sirocco_ion_rates;

/* populate_ion_rate_matrix on the GPU for ncell cells at electron densities
   ne[c] and neutral / ionised hydrogen densities nh1[c], nh2[c].  The
   reference's matrix is block-diagonal by element; A receives each cell's
   element blocks one after another (row-major, elem_n[e]^2 each, elements in
   order), b each cell's nions right-hand side.  Every entry is bit-identical
   to the reference's.  Tables whose rates reach outside an element's block (a
   charge-exchange term above a neutral ion with a nonzero rate, an ionisation
   or inner-shell yield past the element's last ion) return SIROCCO_EINVAL.
   Host arrays. */
int ion_rate_matrices_batched(const sirocco_ion_table *tab, int ncell, const sirocco_ion_rates *rates,
                              const double *ne, const double *nh1, const double *nh2, double *A, double *b);

/* A macro-atom model as calc_matom_matrix (source/macro_accelerate.c:31-348)
   walks it.  Level u's jumps, each list in the reference's order, are entries
   [x_start[u], x_start[u+1]) of the matching target arrays: downward
   bound-bound (bbd: the line's lower level), Auger (aug: target level and
   Avalue_auger * branching_ratio), downward bound-free (bfd: the continuum's
   lower level), upward bound-bound (bbu: the line's upper level), upward
   bound-free (bfu: the continuum's upper level).  The k-packet row takes the
   macro lines' (kbb) and macro continua's (kbf) upper levels, in line and
   continuum order.  Host arrays. */
typedef struct sirocco_matom_table {
  int nlev;                                   /* nlevels_macro; the k-packet is row and column nlev */
  const double *ex;                           /* [nlev] level energies */
  const int *bbd_start, *bbd_target;          /* [nlev + 1], [bbd_start[nlev]] */
  const int *aug_start, *aug_target;
  const double *aug_rate;
  const int *bfd_start, *bfd_target;
  const int *bbu_start, *bbu_target;
  const int *bfu_start, *bfu_target;
  int n_kbb, n_kbf;
  const int *kbb_target, *kbf_target;
} sirocco_matom_table;

/* Per-cell coefficients, cell after cell, one per jump of the matching list:
   bbd_rad = a21 * p_escape and bbd_coll = q21; bfd_sp = recomb_sp and bfd_qrec
   = q_recomb; bbu_rad = b12 * jbar and bbu_coll = q12; bfu_gamma, bfu_alpha
   (alpha_st), bfu_ratio (upper / lower level density, zero below
   DENSITY_PHOT_MIN) and bfu_qion = q_ioniz; kbb / kbf the cooling rates of the
   macro lines / continua (cooling_bb, cooling_bf_col); kr the k-packet to
   r-packet rate summed as the reference sums it; ne the electron density (one
   per cell). */
typedef struct sirocco_matom_rates {
  const double *bbd_rad, *bbd_coll, *bfd_sp, *bfd_qrec, *bbu_rad, *bbu_coll;
  const double *bfu_gamma, *bfu_alpha, *bfu_ratio, *bfu_qion, *kbb, *kbf, *kr, *ne;
} sirocco_matom_rates;

/* The Q / R assembly and normalisation of calc_matom_matrix
   (macro_accelerate.c:82-284) on the GPU for ncell cells: N = I - Q / Q_norm,
   (nlev + 1)^2 row-major per cell, and the diagonal of R / Q_norm, nlev + 1
   per cell, each bit-identical to the reference's.  N and R may be host or
   device pointers; device outputs feed matom_matrices_batched directly.
   Targets outside 0..nlev-1 return SIROCCO_EINVAL. */
int matom_rate_matrices_batched(const sirocco_matom_table *tab, int ncell, const sirocco_matom_rates *rates,
                                double *N, double *R);

/* ion_populations_lockstep with the rate matrices assembled on the GPU from
   `tab` and `rates` each round (only n_e and the hydrogen densities change
   between rounds), so no matrix crosses the bus.  Same outputs and rules. */
int ion_populations_lockstep_rates(const sirocco_ion_table *tab, int ncell, const sirocco_ion_rates *rates,
                                   int h_elem, const double *elem_dens, double *ne, double *den, int *status,
                                   int *iters);

/* Macro-atom level populations of one macro element for ncell cells at once:
   the loop of macro_pops (source/macro_gov.c:336-505), one batched solve per
   round over every unfinished cell.  The element has n levels in matrix order
   (the reference's conf_to_matrix already applied) and nion ions, ion q owning
   levels ion_first[q] .. ion_first[q]+ion_nlte[q]-1; g[n] are the levels'
   statistical weights and radiative[lo*n+up] != 0 marks a radiative link
   between levels lo < up.  scale[c] turns a cell's fractional ion population
   into a density (ele[].abun * rho * rho2nh).  Each round the library calls
   `assemble` for the unfinished cells: it fills each listed cell's n x n rate
   matrix (macro_pops_fill_rate_matrix) into A, cell after cell, using dilute
   estimators when attempt[i] > 1 (get_dilute_estimators after a numerical
   error).  The library then replaces the first row with ones, solves with
   b = e_0, zeroes populations below DENSITY_MIN, clears population inversions
   (upper > lower * g_up / g_lo * 0.999999 on linked levels, macro_gov.c:771),
   and accepts the cell unless an ion density or level population is negative or
   non-finite (:823); a singular system gives the reference's zero populations.
   pop[c*n + k] receives the accepted populations; status[c] is 0, or -2 when
   200 rounds never produced acceptable populations; iters[c] counts rounds.
   All arrays are host arrays. */
typedef int (*sirocco_macro_assemble_fn)(void *user, int ncell, const int *cells, const int *attempt, double *A);
int macro_pops_lockstep(int ncell, int n, int nion, const int *ion_first, const int *ion_nlte, const double *g,
                        const unsigned char *radiative, const double *scale, sirocco_macro_assemble_fn assemble,
                        void *user, double *pop, int *status, int *iters);

/* Macro-atom jumping matrices of a whole cycle (the reference's
   calc_matom_matrix, source/macro_accelerate.c:311-334, called per cell from
   calc_all_matom_matrices :1054-1061).  For every cell s, N_s = I - Q/Q_norm
   (n[s] x n[s], row-major at offA[s]) is inverted in the precision mode of
   sirocco_set_precision -- GSL-exactly in SIROCCO_FP64; in SIROCCO_FAST by the
   certified kernel when N_s passes its M-matrix certificate, B and C then
   formed inside that kernel -- and
   B_s = N_s^-1 diag(R_s) is written at offA[s] of B, with R_s the n[s] diagonal
   entries of R at offv[s].  C, which may be null, receives the row running
   totals of B (C[r][c] = B[r][0] + ... + B[r][c], summed left to right as
   matom_deactivation_from_matrix, :995-1008, sums them), so that a draw is a
   search of one row of C.  status[s] is invert_matrix's code; a singular cell
   gets B = C = 0, as the reference's zero-filled inverse buffer gives.  Layout
   arrays are host arrays; N, R, B, C and status are all host or all device
   pointers (device: B and C can stay resident for matom_sample_batched). */
int matom_matrices_batched(int nsys, const int *n, const int64_t *offA, const int64_t *offv, const double *N,
                           const double *R, double *B, double *C, int *status);

/* Batched draws of the macro-atom deactivation (matom_deactivation_from_matrix,
   source/macro_accelerate.c:951-1018) from the running totals C of
   matom_matrices_batched: query i activates level level[i] of cell sys[i] with
   the uniform number z[i] and gets target[i] = 0 if z <= 0, else the first
   column whose running total is not below z; -1 if the row total stays below z
   (where the reference's loop would read past the row), -2 for a cell or level
   out of range.  n and offA are the host layout arrays of C; C, sys, level, z
   and target are all host or all device pointers. */
int matom_sample_batched(int nq, int nsys, const int *n, const int64_t *offA, const double *C, const int *sys,
                         const int *level, const double *z, int *target);

/* No counterpart in the reference.  Batched solve that allocates no memory at
   all, for callers that cannot let a library allocate on the GPU: host codes
   that reserve the device's memory up front for their own arena (a cudaMalloc
   from a library then fails, or eats the budget of the other MPI ranks sharing
   the GPU), and codes that must not pay the device-wide synchronisation that
   cudaMalloc / cudaFree bring while other streams are busy.  Everything is a
   device pointer, the layout arrays n / offA / offv included; nmax is the
   largest order in the batch, at most SIROCCO_NOALLOC_MAX_N (larger returns
   SIROCCO_ESIZE; a system above nmax gets status -1).  Results and codes are
   those of solve_matrix_batched (GSL-exact FP64).  The factorisation scratch is
   a static device array of SIROCCO_NOALLOC_SLABS x MAX_N^2 doubles (16 MiB)
   that every GPU loading this library holds until exit; its address is looked
   up on the first call on each device.  All calls share that array, so calls
   whose work overlaps on the GPU (other streams, other host threads) race:
   serialise them.  The call only enqueues work on `stream`. */
#define SIROCCO_NOALLOC_MAX_N 512
#define SIROCCO_NOALLOC_SLABS 8
int solve_matrix_batched_noalloc(int nsys, int nmax, const int *n, const int64_t *offA, const double *A,
                                 const int64_t *offv, const double *b, double *x, int *status, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* SIROCCO_SOLVE_H */
