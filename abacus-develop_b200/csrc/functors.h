// Launchers for the DEVICE_GPU op-functor bodies (functors.cu).
#pragma once
#include <cuda_runtime.h>

#include "common.h"
#include "fft_core.cuh"

namespace b200 {

template <typename T, typename R>
void ekinetic_pw(int nband, int npw, int max_npw, R tpiba2, const R* gk2, T* hpsi, const T* psi, cudaStream_t s);
template <typename T, typename R> void veff_pw(long size, T* out, const R* in, cudaStream_t s);
template <typename T, typename R> void veff_pw_npol2(long size, T* out, T* out1, const R* const in[4], cudaStream_t s);
template <typename T, typename R>
void nonlocal_pw(int l1, int l2, int l3, int& sum, int& iat, int spin, int nkb, int dx, int dy, int dz, const R* deeq,
                 T* ps, const T* becp, cudaStream_t s);
template <typename T>
void nonlocal_pw_nc(int l1, int l2, int l3, int& sum, int& iat, int nkb, int dx, int dy, int dz, const T* dnc, T* ps,
                    const T* becp, cudaStream_t s);
template <typename T> void set_3d_fft_box(int npwk, const int* idx, const T* in, T* out, cudaStream_t s);
template <typename T, typename R>
void set_recip_to_real_output(long nrxx, int add, R factor, const T* in, T* out, cudaStream_t s);
template <typename T, typename R>
void set_real_to_recip_output(int npw, long nxyz, int add, R factor, const int* idx, const T* in, T* out, cudaStream_t s);

}  // namespace b200
