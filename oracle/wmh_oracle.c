/*
 * CPU oracle for the weighted-minhash hash path.  TEST INFRASTRUCTURE ONLY:
 * tests, the smoke check and the CPU-baseline leg of the benchmark load this
 * file's library as the checker.  The product never links it.
 *
 * It restates, in plain C, the arithmetic of the reference CUDA kernel
 * `weighted_minhash_cuda` (kernel.cu:56-112 of src-d/minhashcuda):
 *
 *   w      = logf(weight)                                   kernel.cu:95
 *   t      = floorf(w / r + beta)                           kernel.cu:103
 *   ln_y   = (t - beta) * r                                 kernel.cu:104
 *   ln_a   = ln_c - ln_y - r                                kernel.cu:105
 *   keep (col, (uint32)(int32)t) of the strict-'<' argmin   kernel.cu:106-109
 *   running minimum starts at FLT_MAX                       kernel.cu:79
 *
 * and the parameter-initialisation arithmetic of kernel.cu:18-36 together with
 * the draw order of minhashcuda.cc:179-200.
 *
 * Two details are spelled out because the reference leaves them to nvcc:
 *  - form 1 ("fused"): ln_a = fmaf(-(t - beta), r, ln_c) - r, i.e. the
 *    multiply of line 104 contracted into the subtraction of line 105;
 *    form 0 ("unfused"): every operation rounded on its own.  Which form the
 *    reference build uses is pinned by running it on the GPU (tests).
 *  - the float->int32 conversion of t follows the GPU's saturating rule
 *    (NaN -> 0, clamp to [INT32_MIN, INT32_MAX]); C leaves it undefined.
 *
 * A (row, sample) with no entry below FLT_MAX (an empty row, zero or negative
 * or NaN weights) has no defined output in the reference (it writes stale
 * data, kernel.cu:81-87).  The oracle writes (0xFFFFFFFF, 0xFFFFFFFF) there,
 * the byte pattern the reference's debug build pre-fills its output with
 * (minhashcuda.cc:420-424); the CUDA engine does the same.
 *
 * Build: see oracle/Makefile (-O3 -ffp-contract=off: no contraction except
 * the explicit fmaf of form 1).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define WMH_NONE 0xFFFFFFFFu

/* GPU float->int32 conversion (cvt.rzi.s32.f32): truncate, saturate, NaN->0. */
static inline int32_t gpu_f2i(float t) {
  if (t != t) return 0;
  if (t >= 2147483648.0f) return INT32_MAX;
  if (t < -2147483648.0f) return INT32_MIN;
  return (int32_t)t;
}

/* Parameters re-laid as [dim][3][samples] so the per-nnz sweep is contiguous. */
typedef struct {
  uint32_t dim;
  uint32_t samples;
  float *p; /* [dim][3][samples]: r, ln_c, beta */
} wmh_oracle_params;

/* rs/ln_cs/betas are the C-ABI layout: row-major [samples][dim]
 * (minhashcuda.h:84-103). */
wmh_oracle_params *wmh_oracle_prepare(const float *rs, const float *ln_cs,
                                      const float *betas, uint32_t dim,
                                      uint32_t samples) {
  wmh_oracle_params *h = (wmh_oracle_params *)malloc(sizeof(*h));
  if (!h) return NULL;
  h->dim = dim;
  h->samples = samples;
  h->p = (float *)malloc((size_t)dim * 3 * samples * sizeof(float));
  if (!h->p) {
    free(h);
    return NULL;
  }
  #pragma omp parallel for schedule(static)
  for (int64_t d = 0; d < (int64_t)dim; d++) {
    float *col = h->p + (size_t)d * 3 * samples;
    for (uint32_t s = 0; s < samples; s++) {
      size_t i = (size_t)s * dim + (size_t)d;
      col[s] = rs[i];
      col[samples + s] = ln_cs[i];
      col[2 * samples + s] = betas[i];
    }
  }
  return h;
}

void wmh_oracle_release(wmh_oracle_params *h) {
  if (h) {
    free(h->p);
    free(h);
  }
}

/* Hash rows [0, length) of a CSR block.  rows[] holds absolute offsets into
 * weights/cols (rows[0] need not be 0, as in minhashcuda.cc:447-452).
 * lnw, if not NULL, supplies ln(weight) per nnz (indexed like weights) so the
 * check can use the GPU's own logf values.  Output: [length][samples][2]. */
int wmh_oracle_hash(const wmh_oracle_params *h, const float *weights,
                    const float *lnw, const uint32_t *cols,
                    const uint32_t *rows, uint32_t length, int form,
                    int nthreads, uint32_t *output) {
  if (!h || !weights || !cols || !rows || !output) return 1;
  const uint32_t S = h->samples;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  #pragma omp parallel
  {
    float *mn = (float *)malloc(S * sizeof(float));
    float *tf = (float *)malloc(S * sizeof(float));
    uint32_t *kk = (uint32_t *)malloc(S * sizeof(uint32_t));
    #pragma omp for schedule(dynamic, 64)
    for (int64_t row = 0; row < (int64_t)length; row++) {
      for (uint32_t s = 0; s < S; s++) {
        mn[s] = FLT_MAX;
        kk[s] = WMH_NONE;
        tf[s] = 0.0f;
      }
      for (uint32_t i = rows[row]; i < rows[row + 1]; i++) {
        const float w = lnw ? lnw[i] : logf(weights[i]);
        const uint32_t d = cols[i];
        if (d >= h->dim) continue; /* the engine reports such input as invalid */
        const float *col = h->p + (size_t)d * 3 * S;
        const float *rr = col, *cc = col + S, *bb = col + 2 * S;
        if (form) {
          for (uint32_t s = 0; s < S; s++) {
            const float r = rr[s], b = bb[s];
            const float t = floorf(w / r + b);
            const float ln_a = fmaf(-(t - b), r, cc[s]) - r;
            if (ln_a < mn[s]) {
              mn[s] = ln_a;
              kk[s] = d;
              tf[s] = t;
            }
          }
        } else {
          for (uint32_t s = 0; s < S; s++) {
            const float r = rr[s], b = bb[s];
            const float t = floorf(w / r + b);
            const float ln_y = (t - b) * r;
            const float ln_a = (cc[s] - ln_y) - r;
            if (ln_a < mn[s]) {
              mn[s] = ln_a;
              kk[s] = d;
              tf[s] = t;
            }
          }
        }
      }
      uint32_t *out = output + (size_t)row * S * 2;
      for (uint32_t s = 0; s < S; s++) {
        out[2 * s] = kk[s];
        out[2 * s + 1] = kk[s] == WMH_NONE ? WMH_NONE : (uint32_t)gpu_f2i(tf[s]);
      }
    }
    free(mn);
    free(tf);
    free(kk);
  }
  return 0;
}

/* Parameter arithmetic of kernel.cu:18-36 applied in the order of
 * minhashcuda.cc:186-200 to five uniform streams u1..u5 of n floats:
 *   rs = -logf(u2 * u1); ln_cs = logf(-logf(u3 * u4)); betas = u5.
 * Uses the host logf, so it matches the GPU only up to logf's rounding. */
void wmh_oracle_params_from_uniforms(const float *u1, const float *u2,
                                     const float *u3, const float *u4,
                                     const float *u5, uint64_t n, float *rs,
                                     float *ln_cs, float *betas) {
  #pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) {
    rs[i] = -logf(u2[i] * u1[i]);
    const float g = -logf(u3[i] * u4[i]);
    ln_cs[i] = logf(g);
    betas[i] = u5[i];
  }
}

/* Host logf over an array (the tests compare it with the GPU's logf). */
void wmh_oracle_logf(const float *x, float *y, uint64_t n) {
  for (uint64_t i = 0; i < n; i++) y[i] = logf(x[i]);
}
