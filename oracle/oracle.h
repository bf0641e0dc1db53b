// Oracle C ABI -- TEST INFRASTRUCTURE ONLY (see nlsar_oracle.cpp header).
#ifndef DESPECKCL_B200_ORACLE_H
#define DESPECKCL_B200_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

// One (patch, scale) entry of an NL-SAR statistics collection, the fields of
// nlsar::stats (include/compute/nlsar/stats.h:28-55 in the reference).
typedef struct oracle_lut {
  int patch_size;
  int scale_size;
  unsigned int lut_size;
  float dissims_min;
  float dissims_max;
  const float* quantilles;
  const float* chi2cdf_inv;
} oracle_lut;

int oracle_nlsar_insar(const float* a1, const float* a2, const float* ph, float* ref, float* phase, float* coh,
                       int H, int W, int sws, const int* patches, int np, const int* scales, int ns,
                       const oracle_lut* luts, int nluts, float h, float c, int select_mode, int use_double,
                       int tile_h, int tile_w, int nthreads, int* sel, double* bin_margin, double* enl_margin,
                       double* var_cond, double* kappa, double* bin_margin_all);
int oracle_nlsar_covmat(const float* cin, float* cout, int H, int W, int dim, int sws, const int* patches, int np,
                        const int* scales, int ns, const oracle_lut* luts, int nluts, float h, float c,
                        int select_mode, int use_double, int tile_h, int tile_w, int nthreads);
float oracle_pixel_similarity_3x3(const float* a, const float* b);
float oracle_rescale_gamma_dim(int dim);
int oracle_overlap(int sws, const int* patches, int np, const int* scales, int ns);

// training: dissimilarities and LUTs
long oracle_training_dissims(const float* cov, int H, int W, int dim, int patch, int scale, float* out, long cap);
int oracle_stats_from_dissims(const float* dissims, long n, unsigned lut_size, float* dmin, float* dmax,
                              float* quantilles, float* chi2cdf_inv);
double oracle_chi2_inv(double y, double nu);
int oracle_nlsar_training_insar(const float* a1, const float* a2, const float* ph, int H, int W,
                                const int* patches, int np, const int* scales, int ns, int* out_patch,
                                int* out_scale, float* out_dmin, float* out_dmax, float* out_quant,
                                float* out_chi2);

// Goldstein filter, one tile (goldstein_oracle.cpp)
int oracle_goldstein(const float* a1, const float* a2, const float* phi, float* ref, float* phase, int H, int W,
                     int patch_size, int overlap, float alpha, int use_double);
int oracle_goldstein_tile_side(int H, int W, int patch_size, int overlap);

// NL-InSAR (nlinsar_oracle.cpp)
float oracle_nlinsar_h_theo(int patch_size);
int oracle_nlinsar(const float* a1, const float* a2, const float* ph, float* ref, float* phase, float* coh, int H,
                   int W, int sws, int patch_size, int niter, int lmin, int use_double, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
