/*
 * Seeded synthetic graphs, plain C -- TEST INFRASTRUCTURE ONLY (see gen.c).
 * Produces the same CSR arrays as the library's cgp_gen_rmat / cgp_gen_grid /
 * cgp_gen_chung_lu / cgp_gen_weights / cgp_pick_sources.
 */
#ifndef CGP_ORACLE_GEN_H
#define CGP_ORACLE_GEN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_W_NONE 0
#define ORACLE_W_U32 1
#define ORACLE_W_F32 2

/* Host CSR owned by this library (free with oracle_csr_free). */
typedef struct {
  int64_t V;
  int64_t E;
  int64_t* row;
  int32_t* col;
  void* w;             /* uint32 or float per entry, or NULL */
  int32_t weight_kind; /* ORACLE_W_* */
  int32_t reserved;
} oracle_csr;

/* All return 0 on success, 1 for invalid arguments, 2 when out of memory. */
int oracle_csr_from_edges(int64_t V, int64_t M, const int32_t* src, const int32_t* dst,
                          int32_t symmetrize, oracle_csr* out);
int oracle_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b, double c,
                    uint64_t seed, int32_t permute, oracle_csr* out);
int oracle_gen_grid(int32_t rows, int32_t cols, double delete_frac, double shortcut_frac,
                    uint64_t seed, oracle_csr* out);
int oracle_gen_chung_lu(int64_t V, double exponent, double mean_degree, uint64_t seed,
                        oracle_csr* out);
int oracle_gen_weights(oracle_csr* g, int32_t kind, double p0, double p1, int32_t lognormal,
                       uint64_t seed);
int oracle_pick_sources(const oracle_csr* g, int32_t count, int32_t min_degree,
                        const uint8_t* allowed, uint64_t seed, int32_t* sources);
void oracle_csr_free(oracle_csr* g);

#ifdef __cplusplus
}
#endif

#endif
