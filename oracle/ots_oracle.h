/*
 * ots_oracle.h -- CPU oracle interface (test infrastructure only; see
 * ots_oracle.c).  Stencil numbering matches include/ots.h.
 */
#ifndef OTS_ORACLE_H
#define OTS_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  ORC_JACOBI_1D = 0,
  ORC_JACOBI_1D_5PT,
  ORC_JACOBI_1D_7PT,
  ORC_JACOBI_2D,
  ORC_JACOBI_3D,
  ORC_POISSON_2D,
  ORC_POISSON_3D,
  ORC_GRADIENT_2D,
  ORC_GRADIENT_3D,
  ORC_FDTD_2D,
  ORC_RICIAN_2D,
  ORC_TV_UPDATE_2D,
  ORC_CS_3D,
  ORC_NUM_STENCILS
};

enum { ORC_VARIANT_BASELINE = 0, ORC_VARIANT_REF = 1 };

typedef struct {
  int dims;
  int padding;
  int padded_size;
  int real_size;
  int size_lcm;
  int comps[3];
  int rpb[3];
  int num_blocks[3];
  int shared[3];
} orc_geometry;

int orc_set_threads(int n);
int orc_dims(int stencil);
int orc_num_state(int stencil);
int orc_num_aux(int stencil);
int orc_radius(int stencil);
float orc_default_coef(int stencil, int variant);

int orc_geometry_ref(int stencil, int n, int T, int bx, int by, int bz, int E, orc_geometry* g);

void orc_fill_ref_1d_runner(int P, int lo, int hi, unsigned seed, float* out);
void orc_fill_ref(int dims, int P, int lo, int hi, unsigned seed, float** fields, int nfields);

void orc_sweep_f32(int stencil, int variant, int dims, int P, int lo, int hi, float coef,
                   float h2, int steps, int t0, float** state, float* const* aux);
void orc_sweep_f64(int stencil, int variant, int dims, int P, int lo, int hi, float coef,
                   float h2, int steps, int t0, double** state, double* const* aux);

int orc_compare(int dims, int P, int lo, int hi, const float* host, const float* device,
                double* error_norm, double* ref_norm);
void orc_error_vs_f64(int dims, int P, int lo, int hi, const float* got, const double* ref,
                      double floor, double* max_rel, double* rms);

#ifdef __cplusplus
}
#endif

#endif
