/*
 * CPU restatement of AD-TLERT's normal-sensitivity contraction (TEST INFRASTRUCTURE ONLY:
 * the checker and the timed CPU baseline, never part of the product).
 *
 *   out[d][c] = -sum_w sum_i sum_j (u_M - u_N)[i] * T[w][c][i][j] * (u_A - u_B)[j]
 *
 * over the K dofs of cell c, accumulated per entry in the fixed (w, i, j) order of the
 * reference kernel (adtlert/forward/kernels.py:138-177); field row S (one past the last) is a
 * remote electrode with zero potential. Rows are split over `threads` POSIX threads.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>

typedef struct {
  const double* phi;
  const int32_t *a, *b, *m, *n, *cells;
  const double* templates;
  double* out;
  int W, S, D, C, K, d0, d1;
  int64_t N;
} job_t;

static inline double potential(const double* field, int row, int S, int64_t N, int node) {
  return row < S ? field[(int64_t)row * N + node] : 0.0;
}

static void* run(void* arg) {
  const job_t* j = (const job_t*)arg;
  for (int d = j->d0; d < j->d1; ++d) {
    for (int c = 0; c < j->C; ++c) {
      const int32_t* nodes = j->cells + (int64_t)c * j->K;
      double acc = 0.0;
      for (int w = 0; w < j->W; ++w) {
        const double* field = j->phi + (int64_t)w * j->S * j->N;
        const double* t = j->templates + ((int64_t)w * j->C + c) * j->K * j->K;
        double current[16];
        for (int q = 0; q < j->K; ++q)
          current[q] = potential(field, j->a[d], j->S, j->N, nodes[q]) - potential(field, j->b[d], j->S, j->N, nodes[q]);
        for (int i = 0; i < j->K; ++i) {
          const double receiver =
              potential(field, j->m[d], j->S, j->N, nodes[i]) - potential(field, j->n[d], j->S, j->N, nodes[i]);
          for (int q = 0; q < j->K; ++q) acc += receiver * (t[i * j->K + q] * current[q]);
        }
      }
      j->out[(int64_t)d * j->C + c] = -acc;
    }
  }
  return NULL;
}

void normal_sensitivity_cpu(const double* phi, const int32_t* a, const int32_t* b, const int32_t* m,
                            const int32_t* n, const int32_t* cells, const double* templates,
                            double* out, int W, int S, int64_t N, int D, int C, int K, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  pthread_t tid[256];
  job_t jobs[256];
  for (int t = 0; t < threads; ++t) {
    job_t j = {phi, a, b, m, n, cells, templates, out, W, S, D, C, K,
               (int)((int64_t)D * t / threads), (int)((int64_t)D * (t + 1) / threads), N};
    jobs[t] = j;
    pthread_create(&tid[t], NULL, run, &jobs[t]);
  }
  for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
}
