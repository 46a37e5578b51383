// Sampling and harmonic-index helpers of the drop-in C ABI.  Same names,
// arguments, results and error behaviour as the reference's
// src/c/so3_sampling.c (line numbers in include/so3/so3_sampling.h); callers
// size their buffers with these, so they must agree exactly.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>

#include "so3/so3_sampling.h"

typedef std::complex<double> cd;

static void so3_die(const char* msg, const char* fn) {
  printf("ERROR: %s.\n", msg);
  printf("ERROR: Occurred in function <%s> of file %s.\n", fn, __FILE__);
  exit(1);
}
#define DIE(msg) so3_die(msg, __func__)

extern "C" {

cd so3_sampling_weight(const so3_parameters_t* p, int q) {
  if (p->sampling_scheme != SO3_SAMPLING_MW && p->sampling_scheme != SO3_SAMPLING_MW_SS)
    DIE("Invalid sampling scheme.");
  if (q == 1) return cd(0.0, -SO3_PION2);
  if (q == -1) return cd(0.0, SO3_PION2);
  if (q % 2 == 0) return cd(2.0 / (1.0 - (double)q * q), 0.0);
  return cd(0.0, 0.0);
}

int so3_sampling_nalpha(const so3_parameters_t* p) {
  switch (p->sampling_scheme) {
    case SO3_SAMPLING_MW: return 2 * p->L - 1;
    case SO3_SAMPLING_MW_SS: return 2 * p->L;
    default: DIE("Invalid sampling scheme.");
  }
  return 0;
}

int so3_sampling_nbeta(const so3_parameters_t* p) {
  switch (p->sampling_scheme) {
    case SO3_SAMPLING_MW: return p->L;
    case SO3_SAMPLING_MW_SS: return p->L + 1;
    default: DIE("Invalid sampling scheme.");
  }
  return 0;
}

int so3_sampling_ngamma(const so3_parameters_t* p) { return p->steerable ? p->N : 2 * p->N - 1; }

int so3_sampling_f_size(const so3_parameters_t* p) {
  return so3_sampling_nalpha(p) * so3_sampling_nbeta(p) * so3_sampling_ngamma(p);
}

int so3_sampling_n(const so3_parameters_t* p) {
  const int L = p->L;
  switch (p->sampling_scheme) {
    case SO3_SAMPLING_MW: return ((2 * L - 1) * (L - 1) + 1) * so3_sampling_ngamma(p);
    case SO3_SAMPLING_MW_SS: return ((2 * L) * (L - 1) + 2) * so3_sampling_ngamma(p);
    default: DIE("Invalid sampling scheme.");
  }
  return 0;
}

double so3_sampling_a2alpha(int a, const so3_parameters_t* p) {
  switch (p->sampling_scheme) {
    case SO3_SAMPLING_MW: return 2.0 * a * SO3_PI / (2.0 * p->L - 1.0);
    case SO3_SAMPLING_MW_SS: return 2.0 * a * SO3_PI / (2.0 * p->L);
    default: DIE("Invalid sampling scheme.");
  }
  return 0.0;
}

double so3_sampling_b2beta(int b, const so3_parameters_t* p) {
  switch (p->sampling_scheme) {
    case SO3_SAMPLING_MW: return (2.0 * b + 1.0) * SO3_PI / (2.0 * p->L - 1.0);
    case SO3_SAMPLING_MW_SS: return 2.0 * b * SO3_PI / (2.0 * p->L);
    default: DIE("Invalid sampling scheme.");
  }
  return 0.0;
}

double so3_sampling_g2gamma(int g, const so3_parameters_t* p) {
  if (p->steerable) return g * SO3_PI / p->N;
  return 2.0 * g * SO3_PI / (2.0 * p->N - 1.0);
}

int so3_sampling_flmn_size(const so3_parameters_t* p) {
  const int L = p->L, N = p->N;
  switch (p->storage) {
    case SO3_STORAGE_PADDED: return p->reality ? N * L * L : (2 * N - 1) * L * L;
    case SO3_STORAGE_COMPACT:
      // sum_{n=1}^{N-1} n^2 = (N-1) N (2N-1) / 6
      return p->reality ? N * (6 * L * L - (N - 1) * (2 * N - 1)) / 6 : (2 * N - 1) * (3 * L * L - N * (N - 1)) / 3;
    default: DIE("Invalid storage method.");
  }
  return 0;
}

void so3_sampling_elmn2ind(int* ind, int el, int m, int n, const so3_parameters_t* p) {
  const int L = p->L, N = p->N, an = abs(n);
  int off;
  switch (p->storage) {
    case SO3_STORAGE_PADDED:
      switch (p->n_order) {
        case SO3_N_ORDER_ZERO_FIRST: off = (n < 0 ? -2 * n - 1 : 2 * n) * L * L; break;
        case SO3_N_ORDER_NEGATIVE_FIRST: off = (N - 1 + n) * L * L; break;
        default: DIE("Invalid n-order.");
      }
      *ind = off + el * el + el + m;
      return;
    case SO3_STORAGE_COMPACT:
      if (an > el) DIE("Tried to access component with n > l in compact storage.");
      switch (p->n_order) {
        case SO3_N_ORDER_ZERO_FIRST:
          off = (2 * an - 1) * (3 * L * L - an * (an - 1)) / 3;
          if (n >= 0) off += L * L - n * n;
          break;
        case SO3_N_ORDER_NEGATIVE_FIRST:
          off = (N - 1 + n) * L * L - (2 * N - 1) * (N - 1) * N / 6;
          if (n <= 0)
            off += an * (2 * an + 1) * (an + 1) / 6;
          else
            off -= an * (2 * an - 1) * (an - 1) / 6;
          break;
        default: DIE("Invalid n-order.");
      }
      *ind = off + el * el - n * n + el + m;
      return;
    default: DIE("Invalid storage method.");
  }
}

void so3_sampling_ind2elmn(int* el, int* m, int* n, int ind, const so3_parameters_t* p) {
  const int L = p->L, N = p->N;
  switch (p->storage) {
    case SO3_STORAGE_PADDED: {
      const int blk = ind / (L * L);
      switch (p->n_order) {
        case SO3_N_ORDER_ZERO_FIRST: *n = (blk % 2) ? -(blk + 1) / 2 : blk / 2; break;
        case SO3_N_ORDER_NEGATIVE_FIRST: *n = blk - (N - 1); break;
        default: DIE("Invalid n-order.");
      }
      ind %= L * L;
      break;
    }
    case SO3_STORAGE_COMPACT: {
      int off;
      switch (p->n_order) {
        case SO3_N_ORDER_ZERO_FIRST:
          *n = 0;
          off = 0;
          while (ind + off >= L * L) {
            ind -= L * L - off;
            if (*n >= 0) {
              *n = -(*n + 1);
              off = (*n) * (*n);
            } else {
              *n = -(*n);
            }
          }
          break;
        case SO3_N_ORDER_NEGATIVE_FIRST:
          *n = -N + 1;
          off = (*n) * (*n);
          while (ind + off >= L * L) {
            ind -= L * L - off;
            (*n)++;
            off = (*n) * (*n);
          }
          break;
        default: DIE("Invalid n-order.");
      }
      ind += off;
      break;
    }
    default: DIE("Invalid storage method.");
  }
  *el = (int)std::sqrt((double)ind);
  *m = ind - (*el) * (*el) - *el;
}

void so3_sampling_elmn2ind_real(int* ind, int el, int m, int n, const so3_parameters_t* p) {
  if (p->storage != SO3_STORAGE_PADDED && p->storage != SO3_STORAGE_COMPACT) DIE("Invalid storage method.");
  so3_parameters_t q = *p;
  q.n_order = SO3_N_ORDER_NEGATIVE_FIRST;
  int base;
  so3_sampling_elmn2ind(&base, 0, 0, 0, &q);
  so3_sampling_elmn2ind(ind, el, m, n, &q);
  *ind -= base;
}

void so3_sampling_ind2elmn_real(int* el, int* m, int* n, int ind, const so3_parameters_t* p) {
  if (p->storage != SO3_STORAGE_PADDED && p->storage != SO3_STORAGE_COMPACT) DIE("Invalid storage method.");
  so3_parameters_t q = *p;
  q.n_order = SO3_N_ORDER_NEGATIVE_FIRST;
  int base;
  so3_sampling_elmn2ind(&base, 0, 0, 0, &q);
  so3_sampling_ind2elmn(el, m, n, base + ind, &q);
}

void so3_sampling_n_loop_values(int* s, int* e, int* inc, const so3_parameters_t* p) {
  const int N = p->N;
  if (p->reality) {
    switch (p->n_mode) {
      case SO3_N_MODE_ALL:
      case SO3_N_MODE_L: *s = 0, *e = N - 1, *inc = 1; break;
      case SO3_N_MODE_EVEN: *s = 0, *e = ((N - 1) % 2 == 0) ? N - 1 : N - 2, *inc = 2; break;
      case SO3_N_MODE_ODD: *s = 1, *e = ((N - 1) % 2 != 0) ? N - 1 : N - 2, *inc = 2; break;
      case SO3_N_MODE_MAXIMUM: *s = N - 1, *e = N - 1, *inc = 1; break;
      default: DIE("Invalid n-mode.");
    }
  } else {
    switch (p->n_mode) {
      case SO3_N_MODE_ALL:
      case SO3_N_MODE_L: *s = -N + 1, *e = N - 1, *inc = 1; break;
      case SO3_N_MODE_EVEN:
        *s = ((N - 1) % 2 == 0) ? -N + 1 : -N + 2;
        *e = ((N - 1) % 2 == 0) ? N - 1 : N - 2;
        *inc = 2;
        break;
      case SO3_N_MODE_ODD:
        *s = ((N - 1) % 2 != 0) ? -N + 1 : -N + 2;
        *e = ((N - 1) % 2 != 0) ? N - 1 : N - 2;
        *inc = 2;
        break;
      case SO3_N_MODE_MAXIMUM: *s = -N + 1, *e = N - 1, *inc = N > 1 ? 2 * N - 2 : 1; break;
      default: DIE("Invalid n-mode.");
    }
  }
}

void so3_sampling_el_loop_values(int* s, int* e, int* inc, const int n, const so3_parameters_t* p) {
  *s = p->L0 > abs(n) ? p->L0 : abs(n);
  *e = p->n_mode == SO3_N_MODE_L ? abs(n) : p->L - 1;
  *inc = 1;
}

void so3_sampling_m_loop_values(int* s, int* e, int* inc, const int el) {
  *s = -el;
  *e = el;
  *inc = 1;
}

static bool in_range(int i, int s, int e, int inc) { return i >= s && i <= e && (i - s) % inc == 0; }

bool so3_sampling_is_elmn_non_zero(const int el, const int m, const int n, const so3_parameters_t* p) {
  int s, e, inc;
  so3_sampling_n_loop_values(&s, &e, &inc, p);
  if (!in_range(n, s, e, inc)) return false;
  so3_sampling_el_loop_values(&s, &e, &inc, n, p);
  if (!in_range(el, s, e, inc)) return false;
  so3_sampling_m_loop_values(&s, &e, &inc, el);
  return in_range(m, s, e, inc);
}

int so3_sampling_is_elmn_non_zero_return_int(const int el, const int m, const int n, const so3_parameters_t* p) {
  return (int)so3_sampling_is_elmn_non_zero(el, m, n, p);
}

}  // extern "C"
