/* rng_shim.h - stands in for curand_kernel.h when the reference's
 * electron_transport.cu is compiled for oracle pinning.  It defines the
 * header's include guard so the reference's own copy is skipped, and makes
 * curand_init / curand_uniform_double / curand_normal read per-particle
 * injected draws: row `offset` (the reference passes the thread index n as
 * the offset, electron_transport.cu:81) of an n x 8 array; uniforms come
 * from slots 0..3 in call order, normals from slots 4..6 (as float, like
 * curand_normal). */
#pragma once
#define CURAND_KERNEL_H_
__device__ const double *g_shim_draws;
struct curandState { const double *d; int u; int g; };
static __device__ __forceinline__ void curand_init(unsigned long long seed, unsigned long long subseq,
                                                   unsigned long long offset, curandState *s) {
  (void)seed; (void)subseq;
  s->d = g_shim_draws + offset * 8; s->u = 0; s->g = 0;
}
static __device__ __forceinline__ double curand_uniform_double(curandState *s) { return s->d[s->u++]; }
static __device__ __forceinline__ float curand_normal(curandState *s) { return (float)s->d[4 + s->g++]; }
