/*
 * cgc_volume.h -- synthetic benchmark inputs, in a host-only library of their
 * own (libcgcvol.so, no CUDA), so that CPU-only code such as a CPU baseline
 * builds the same workloads without loading the GPU engine.  Status codes are
 * the CGC_* codes of cgc.h.
 *
 * No counterpart in the reference: it reads images and markers from disk
 * (benchmarks/graph_cut/segmentation.cpp:140-151) and ships none.
 */
#ifndef CGC_VOLUME_H
#define CGC_VOLUME_H

#include <stddef.h>
#include <stdint.h>

#include "cgc.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Deterministic capacity volumes for the benchmark workloads (x-fastest,
 * int32): Gaussian spheres (a ball of radius r whose boundary is blurred by a
 * Gaussian of edge_sigma voxels: I = bg + (I_obj-bg)*erfc((d-r)/(sqrt2*sigma))/2)
 * or tubes on a background, Gaussian noise, two-class Gaussian likelihood t-links capS = round(s*(-log p_bg)),
 * capT = round(s*(-log p_fg)) and contrast n-links
 * round(w*exp(-(Ii-Ij)^2/(2*sigma^2))).  nx/ny/nz hold the symmetric n-link
 * to the +x/+y/+z neighbour (0 on the last slice). */
typedef struct cgc_volume_spec {
  int32_t X, Y, Z;
  int32_t kind;              /* 0 = spheres, 1 = tubes */
  uint64_t seed;
  int32_t count;             /* spheres or tubes */
  int32_t n_fixed_radii;     /* spheres: if > 0 use fixed_radii[0..count) */
  double fixed_radii[8];
  double radius_min, radius_max;
  double intensity_min, intensity_max;
  double background, noise_sd;
  double mu_bg, mu_fg, class_sd;
  double tlink_scale, nlink_scale, nlink_sigma;
  int32_t ctrl_min, ctrl_max; /* tubes: control points per spline */
  double edge_sigma;         /* spheres: Gaussian blur of the boundary (voxels), 0 = hard edge */
} cgc_volume_spec;

/* Fills the spec of a named workload: which = 1 (64^3 two spheres),
 * 2 (256^3 40 spheres), 3 (512x512x128 200 tubes), 4 (batched instance
 * `index`, extents in 32..160), 5 (128^3 training instance `index`). */
int cgc_volume_preset(int which, int32_t index, cgc_volume_spec* out);
int cgc_volume_generate(const cgc_volume_spec* spec, int32_t* capS, int32_t* capT,
                        int32_t* nx, int32_t* ny, int32_t* nz, float* image /* may be NULL */);
/* Message of the last failure of these two calls on the calling thread. */
const char* cgc_volume_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* CGC_VOLUME_H */
