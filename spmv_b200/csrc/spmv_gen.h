/* Seeded synthetic workloads (libspmv_gen): matrices in global CSR form
 * (0-based, int32, sorted columns per row) and random vectors.  Host code;
 * no GPU is needed.  Functions returning int give 0 on success, else
 * spmv_gen_last_error() holds the message. */
#ifndef SPMV_GEN_H
#define SPMV_GEN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct spmv_gen_csr_s* spmv_gen_csr;

const char* spmv_gen_last_error(void);

/* out[i] = lo + (hi-lo) * U_i, U_i uniform in [0,1) from (seed, stream, i). */
void spmv_gen_uniform(uint64_t seed, uint64_t stream, double lo, double hi,
                      double* out, int64_t n);
/* out[i] = mean + std * N_i, N_i standard normal from (seed, stream, i). */
void spmv_gen_normal(uint64_t seed, uint64_t stream, double mean, double std,
                     double* out, int64_t n);

int spmv_gen_laplace2d(int64_t nx, int64_t ny, spmv_gen_csr* out);
int spmv_gen_laplace3d(int64_t n, spmv_gen_csr* out);
int spmv_gen_laplace3d_27pt(int64_t n, uint64_t seed, double shift,
                            spmv_gen_csr* out);
int spmv_gen_grid2d_softplus(int64_t nx, int64_t ny, uint64_t seed,
                             double sigma, double shift, spmv_gen_csr* out);
int spmv_gen_knn_laplacian(int64_t n, int k, uint64_t seed, uint64_t sys,
                           double shift, spmv_gen_csr* out);
int spmv_gen_create_a(int64_t N, spmv_gen_csr* out);

int spmv_gen_csr_info(spmv_gen_csr h, int64_t* nrows, int64_t* ncols,
                      int64_t* nnz);
/* Pointers into the handle's arrays, valid until spmv_gen_csr_free. */
int spmv_gen_csr_arrays(spmv_gen_csr h, const int32_t** rowptr,
                        const int32_t** cols, const double** vals);
int spmv_gen_csr_aux(spmv_gen_csr h, double* scalar, const int64_t** i64,
                     int64_t* n_i64, const double** f64, int64_t* n_f64);
void spmv_gen_csr_free(spmv_gen_csr h);

#ifdef __cplusplus
}
#endif

#endif
