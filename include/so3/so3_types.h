/*
 * so3_types.h -- configuration types of the SO3 drop-in C ABI.
 *
 * Binary-compatible with the reference's include/so3/so3_types.h:50-201
 * (enum value order and the eleven 4-byte fields of so3_parameters_t are the
 * contract callers compile against), but self-contained: the reference pulls
 * ssht_dl_method_t from <ssht/ssht.h> (:29); this header defines the same enum
 * (RISBO = 0, TRAPANI = 1, the values the reference's Cython binding declares
 * at src/so3/bindings.pyx:90-91) unless an SSHT header already did.
 */
#ifndef SO3_TYPES
#define SO3_TYPES

#ifdef __cplusplus
#include <complex>
#define SO3_COMPLEX(TYPE) std::complex<TYPE>
extern "C" {
#else
#include <complex.h>
#define SO3_COMPLEX(TYPE) TYPE complex
#endif

#define SO3_PI 3.141592653589793238462643383279502884197
#define SO3_PION2 1.570796326794896619231321691639751442099
#define SO3_SQRT2 1.41421356237309504880168872420969807856967
#define SO3_PROMPT "[so3] "

#if !defined(SO3_SSHT_DL_METHOD_T_DEFINED) && !defined(SSHT_DL_METHOD_DEFINED)
#define SO3_SSHT_DL_METHOD_T_DEFINED
/* Recursion used for the Wigner Delta(pi/2) planes. */
typedef enum { SSHT_DL_RISBO = 0, SSHT_DL_TRAPANI = 1 } ssht_dl_method_t;
#endif

typedef enum {
  SO3_N_ORDER_ZERO_FIRST,     /* n-blocks stored as 0, -1, 1, -2, 2, ... */
  SO3_N_ORDER_NEGATIVE_FIRST, /* n-blocks stored as -N+1, ..., N-1 */
  SO3_N_ORDER_SIZE
} so3_n_order_t;

typedef enum {
  SO3_STORAGE_PADDED,  /* every n-block holds L*L values */
  SO3_STORAGE_COMPACT, /* block n omits l < |n| (L*L - n*n values) */
  SO3_STORAGE_SIZE
} so3_storage_t;

typedef enum {
  SO3_N_MODE_ALL,     /* any n may be non-zero */
  SO3_N_MODE_EVEN,    /* only even n */
  SO3_N_MODE_ODD,     /* only odd n */
  SO3_N_MODE_MAXIMUM, /* only |n| = N-1 */
  SO3_N_MODE_L,       /* only |n| = l */
  SO3_N_MODE_SIZE
} so3_n_mode_t;

typedef enum {
  SO3_SAMPLING_MW,    /* 2L-1 alpha, L beta in (0, pi], 2N-1 gamma */
  SO3_SAMPLING_MW_SS, /* 2L alpha, L+1 beta in [0, pi], 2N-1 gamma */
  SO3_SAMPLING_SIZE
} so3_sampling_t;

/* Zero-initialise before use ("so3_parameters_t p = {0};"). */
typedef struct {
  int verbosity;
  int reality;
  int L0;
  int L;
  int N;
  so3_sampling_t sampling_scheme;
  so3_n_order_t n_order;
  so3_storage_t storage;
  so3_n_mode_t n_mode;
  ssht_dl_method_t dl_method;
  int steerable;
} so3_parameters_t;

#ifdef __cplusplus
}
#endif
#endif
