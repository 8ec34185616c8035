/*
 * splatt.h -- public C interface of the B200 AdaTM library.
 *
 * Drop-in for the SPLATT v1.1.1 / AdaTM public header (reference
 * include/splatt.h). Type widths, enum values and struct layouts are the
 * reference's, so code written against it compiles and links unchanged:
 * indices are 64-bit, values are double, SPLATT_MAX_NMODES is 88. The GPU
 * kernels behind it accept tensors of order 3..8, rank 1..128, dimensions and
 * nonzero counts below 2^32-1; anything else returns SPLATT_ERROR_BADINPUT.
 */
#ifndef ADATM_B200_SPLATT_H
#define ADATM_B200_SPLATT_H

#include <float.h>
#include <inttypes.h>
#include <stdio.h>

/* ---- types (reference include/splatt.h:26-68) ------------------------- */
#define SPLATT_IDX_TYPEWIDTH 64
#define SPLATT_VAL_TYPEWIDTH 64
typedef uint64_t splatt_idx_t;
#define SPLATT_IDX_MAX UINT64_MAX
#define SPLATT_PF_IDX PRIu64
typedef double splatt_val_t;
#define SPLATT_VAL_MIN DBL_MIN
#define SPLATT_VAL_MAX DBL_MAX
#define SPLATT_PF_VAL "f"

#define SPLATT_VER_MAJOR 1
#define SPLATT_VER_MINOR 1
#define SPLATT_VER_SUBMINOR 1

#ifndef SPLATT_MAX_NMODES
#define SPLATT_MAX_NMODES ((splatt_idx_t)88)
#endif

/* ---- options array indices (reference include/splatt.h:93-111) -------- */
typedef enum {
  SPLATT_OPTION_NTHREADS,  /* host threads (ignored by the GPU kernels) */
  SPLATT_OPTION_TOLERANCE, /* stop when |fit - previous fit| < tolerance */
  SPLATT_OPTION_NITER,     /* maximum ALS iterations */
  SPLATT_OPTION_VERBOSITY,
  SPLATT_OPTION_RANDSEED,  /* seed of the factor initialisation */
  SPLATT_OPTION_CSF_ALLOC, /* which trees to build (splatt_csf_type) */
  SPLATT_OPTION_TILE,      /* only SPLATT_NOTILE is supported */
  SPLATT_OPTION_TILEDEPTH,
  SPLATT_OPTION_DECOMP,
  SPLATT_OPTION_COMM,
  SPLATT_OPTION_NOPTIONS
} splatt_option_type;

/* ---- return codes (reference include/splatt.h:117-125) ---------------- */
typedef enum {
  SPLATT_SUCCESS = 1,
  SPLATT_ERROR_BADINPUT,
  SPLATT_ERROR_NOMEMORY
} splatt_error_type;

typedef enum {
  SPLATT_VERBOSITY_NONE,
  SPLATT_VERBOSITY_LOW,
  SPLATT_VERBOSITY_HIGH,
  SPLATT_VERBOSITY_MAX
} splatt_verbosity_type;

typedef enum {
  SPLATT_NOTILE,
  SPLATT_DENSETILE,
  SPLATT_SYNCTILE,
  SPLATT_COOPTILE,
} splatt_tile_type;

/* CSF allocations (reference include/splatt.h:156-164). The three ADAPTIVE
 * values select AdaTM's memoized plan. */
typedef enum {
  SPLATT_CSF_ONEMODE,
  SPLATT_CSF_TWOMODE,
  SPLATT_CSF_ALLMODE,
  SPLATT_ADAPTIVE,
  SPLATT_ADAPTIVE_TIME_EFFICIENT,
  SPLATT_ADAPTIVE_SPACE_EFFICIENT,
} splatt_csf_type;

typedef enum { SPLATT_DECOMP_COARSE, SPLATT_DECOMP_MEDIUM, SPLATT_DECOMP_FINE } splatt_decomp_type;
typedef enum { SPLATT_COMM_POINT2POINT, SPLATT_COMM_ALL2ALL } splatt_comm_type;

static double const SPLATT_VAL_OFF = -DBL_MAX;

/* ---- data structures (reference include/splatt.h:209-287) ------------- */
typedef struct splatt_kruskal {
  splatt_idx_t rank;
  splatt_val_t *factors[SPLATT_MAX_NMODES]; /* row-major dims[m] x rank */
  splatt_val_t *lambda;
  splatt_idx_t nmodes;
  splatt_idx_t dims[SPLATT_MAX_NMODES];
  double fit;
} splatt_kruskal;

typedef struct {
  splatt_idx_t nfibs[SPLATT_MAX_NMODES];
  splatt_idx_t *fptr[SPLATT_MAX_NMODES]; /* fptr[l]: nfibs[l]+1 entries, l <= N-2 */
  splatt_idx_t *fids[SPLATT_MAX_NMODES]; /* fids[0] == NULL for one tile */
  splatt_val_t *vals;                    /* nfibs[N-1] leaf values */
} csf_sparsity;

typedef struct splatt_csf {
  splatt_idx_t nnz;
  splatt_idx_t nmodes;
  splatt_idx_t dims[SPLATT_MAX_NMODES];
  splatt_idx_t dim_perm[SPLATT_MAX_NMODES]; /* dim_perm[l]: mode at level l */
  splatt_tile_type which_tile;
  splatt_idx_t ntiles;
  splatt_idx_t tile_dims[SPLATT_MAX_NMODES];
  csf_sparsity *pt;
} splatt_csf;

/* ---- AdaTM plan structures (reference include/splatt.h:297-358) ------- */
typedef struct rcsf_seq_adaptive {
  splatt_idx_t begin_imten;
  splatt_idx_t n_imten;
  splatt_csf *rcsfs; /* memo trees: tree deg holds level begin_imten-1-deg */
} rcsf_seq_adaptive;

typedef struct group_properties {
  splatt_idx_t memo_mode;
  splatt_idx_t begin_imten;
  splatt_idx_t n_imten;
  splatt_idx_t *o_opt; /* level order of the group's tree */
} group_properties;

typedef struct configurations_adaptive {
  splatt_idx_t n_grp;
  group_properties *grp_prop;
  size_t pspace;
  size_t pops;
  double ptime;
  double rtime;
} configurations_adaptive;

typedef struct pair {
  splatt_idx_t x;
  splatt_idx_t y;
} pair;

#ifdef __cplusplus
extern "C" {
#endif

/* ---- options (reference include/splatt.h:384-398) --------------------- */
double *splatt_default_opts(void);
void splatt_free_opts(double *opts);

/* ---- data structures (reference include/splatt.h:425-467) ------------- */

/* Read a FROSTT-style text tensor (one nonzero per line: N 1-based indices
 * and a value) and build the trees opts[SPLATT_OPTION_CSF_ALLOC] asks for. */
int splatt_csf_load(char const *const fname, splatt_idx_t *nmodes, splatt_csf **tensors,
                    double const *const options);

/* Build the trees of a COO tensor on the GPU (inds[m][n], vals[n]). */
int splatt_csf_convert(splatt_idx_t const nmodes, splatt_idx_t const nnz,
                       splatt_idx_t **const inds, splatt_val_t *const vals,
                       splatt_csf **tensors, double const *const options);

void splatt_free_csf(splatt_csf *tensors, double const *const options);
void splatt_free_kruskal(splatt_kruskal *factored);

/* ---- factorization (reference include/splatt.h:493-497) --------------- */
int splatt_cpd_als(splatt_csf const *const tensors, splatt_idx_t const nfactors,
                   double const *const options, splatt_kruskal *factored);

/* ---- MTTKRP (reference include/splatt.h:519-525) ---------------------- */
int splatt_mttkrp(splatt_idx_t const mode, splatt_idx_t const ncolumns,
                  splatt_csf const *const tensors, splatt_val_t **matrices,
                  splatt_val_t *const matout, double const *const options);

#ifdef __cplusplus
}
#endif

#endif
