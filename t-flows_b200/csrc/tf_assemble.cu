// tf_assemble.cu -- the pressure and momentum matrices assembled on the
// device from face data, through Matrix_Type's pos(1:2, face) map.
//
// Process assembles A % val on the host every outer iteration
// (Compute_Pressure.f90, Rhie_And_Chow.f90:183-205, Compute_Momentum.f90:
// 270-297) and the drop-in then uploads it; with the face data already on
// the device the upload disappears.  Results are bit-identical to the
// reference's face loops:
//
//   * off-diagonals: one thread per face writes its two entries, the
//     reference's assignment (pressure: -a12) or accumulation from the
//     zeroed matrix (momentum: 0 - m12);
//   * diagonals: one thread per cell adds its faces' contributions in
//     ascending face order -- the order in which the reference's sequential
//     face loop reaches that cell -- starting from 0.0, then the terms of
//     the later loops (pressure boundary faces; the inertial term).
//
// Every product and sum is issued as the reference writes it, rounded
// (__dmul_rn, __dadd_rn, ...), with no FMA contraction.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "tf_internal.h"

namespace tf {

__device__ __forceinline__ double fmin_ref(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double fmax_ref(double a, double b) { return (b > a) ? b : a; }

// a12 of Rhie_And_Chow.f90: fc * (fs * v_m(c1) + (1 - fs) * v_m(c2))
__device__ __forceinline__ double p_coef(const double* fc, const double* fw, const double* vm,
                                         int s, int c1, int c2) {
  const double fs = fw[s];
  const double v1 = vm ? vm[c1] : 1.0, v2 = vm ? vm[c2] : 1.0;
  const double t = __dadd_rn(__dmul_rn(fs, v1), __dmul_rn(__dsub_rn(1.0, fs), v2));
  return __dmul_rn(fc[s], t);
}

__global__ void __launch_bounds__(256) k_asm_p_off(int nf, const int* __restrict__ fcell,
                                                   const int* __restrict__ fpos,
                                                   const double* __restrict__ fc,
                                                   const double* __restrict__ fw,
                                                   const double* __restrict__ vm,
                                                   double* __restrict__ val) {
  const int stride = gridDim.x * blockDim.x;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nf; s += stride) {
    const int c1 = fcell[2 * s], c2 = fcell[2 * s + 1];
    if (c2 < 0) continue;
    const double a12 = p_coef(fc, fw, vm, s, c1, c2);
    val[fpos[2 * s]] = -a12;
    val[fpos[2 * s + 1]] = -a12;
  }
}

__global__ void __launch_bounds__(256) k_asm_p_diag(int n, const int* __restrict__ cf_ptr,
                                                    const int* __restrict__ cf,
                                                    const int* __restrict__ fcell,
                                                    const int* __restrict__ dia,
                                                    const double* __restrict__ fc,
                                                    const double* __restrict__ fw,
                                                    const double* __restrict__ vm,
                                                    const int* __restrict__ bnd_open,
                                                    double* __restrict__ val) {
  const int stride = gridDim.x * blockDim.x;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride) {
    double d = 0.0;
    const int e0 = cf_ptr[c], e1 = cf_ptr[c + 1];
    for (int e = e0; e < e1; ++e) {   // interior faces (Rhie_And_Chow.f90:183-205)
      const int s = cf[e] >> 1;
      const int c1 = fcell[2 * s], c2 = fcell[2 * s + 1];
      if (c2 >= 0) d = __dadd_rn(d, p_coef(fc, fw, vm, s, c1, c2));
    }
    if (bnd_open) {                   // boundary faces (Compute_Pressure.f90:140-160)
      for (int e = e0; e < e1; ++e) {
        const int s = cf[e] >> 1;
        if (fcell[2 * s + 1] < 0 && bnd_open[s])
          d = __dadd_rn(d, __dmul_rn(fc[s], vm ? vm[c] : 1.0));
      }
    }
    val[dia[c]] = d;
  }
}

struct MomCoef {
  double m12, m21;
};
// Compute_Momentum.f90:270-297 with blend_matrix: upwind-blended m12, m21
__device__ __forceinline__ MomCoef m_coef(const double* fc, const double* flux, double vis,
                                          double rho, int s) {
  const double m0 = __dmul_rn(vis, fc[s]);
  const double f = flux[s];
  MomCoef k;
  k.m12 = __dsub_rn(m0, __dmul_rn(fmin_ref(f, 0.0), rho));
  k.m21 = __dadd_rn(m0, __dmul_rn(fmax_ref(f, 0.0), rho));
  return k;
}

__global__ void __launch_bounds__(256) k_asm_m_off(int nf, const int* __restrict__ fcell,
                                                   const int* __restrict__ fpos,
                                                   const double* __restrict__ fc,
                                                   const double* __restrict__ flux,
                                                   double vis, double rho,
                                                   double* __restrict__ val) {
  const int stride = gridDim.x * blockDim.x;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < nf; s += stride) {
    if (fcell[2 * s + 1] < 0) continue;
    const MomCoef k = m_coef(fc, flux, vis, rho, s);
    val[fpos[2 * s]] = __dsub_rn(0.0, k.m12);
    val[fpos[2 * s + 1]] = __dsub_rn(0.0, k.m21);
  }
}

__global__ void __launch_bounds__(256) k_asm_m_diag(int n, const int* __restrict__ cf_ptr,
                                                    const int* __restrict__ cf,
                                                    const int* __restrict__ fcell,
                                                    const int* __restrict__ dia,
                                                    const double* __restrict__ fc,
                                                    const double* __restrict__ flux,
                                                    const int* __restrict__ bnd_wall,
                                                    double vis, double rho,
                                                    const double* __restrict__ vol, double dt,
                                                    double* __restrict__ val) {
  const int stride = gridDim.x * blockDim.x;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride) {
    double d = 0.0;
    for (int e = cf_ptr[c]; e < cf_ptr[c + 1]; ++e) {
      const int s = cf[e] >> 1, second = cf[e] & 1;
      const bool interior = fcell[2 * s + 1] >= 0;
      if (!interior && !(bnd_wall && bnd_wall[s])) continue;
      const MomCoef k = m_coef(fc, flux, vis, rho, s);
      d = __dadd_rn(d, second ? k.m21 : k.m12);
    }
    // Inertial_Term.f90 (linear): a0 = rho * vol / dt
    d = __dadd_rn(d, __ddiv_rn(__dmul_rn(rho, vol[c]), dt));
    val[dia[c]] = d;
  }
}

}  // namespace tf

using namespace tf;

extern "C" int tf_faces_register(tf_ctx ctx, tf_matrix m, int n_faces, const int* faces_c,
                                 const int* pos) {
  TF_API_BEGIN
  if (!ctx || !m || m->ctx != ctx || n_faces < 0 || (n_faces > 0 && (!faces_c || !pos)))
    return TF_ERR_ARG;
  const int n = m->nt;
  std::vector<int> fcell((size_t)2 * n_faces + 2), fpos((size_t)2 * n_faces + 2);
  std::vector<int> cnt((size_t)n + 1, 0);
  for (int s = 0; s < n_faces; ++s) {
    const int c1 = faces_c[2 * s], c2 = faces_c[2 * s + 1];
    if (c1 < 1 || c1 > n || c2 > n) return TF_ERR_LAYOUT;
    fcell[2 * s] = c1 - 1;
    fcell[2 * s + 1] = c2 > 0 ? c2 - 1 : -1;
    if (c2 > 0) {
      const int p1 = pos[2 * s], p2 = pos[2 * s + 1];
      if (p1 < 1 || p1 > m->nnz || p2 < 1 || p2 > m->nnz) return TF_ERR_LAYOUT;
      fpos[2 * s] = p1 - 1;
      fpos[2 * s + 1] = p2 - 1;
      ++cnt[c2 - 1];
    } else {
      fpos[2 * s] = fpos[2 * s + 1] = -1;
    }
    ++cnt[c1 - 1];
  }
  // cell -> faces in ascending face order; bit 0: the cell is the face's c2
  std::vector<int> ptr((size_t)n + 1, 0);
  for (int c = 0; c < n; ++c) ptr[c + 1] = ptr[c] + cnt[c];
  std::vector<int> cf((size_t)ptr[n] + 1), fill(ptr.begin(), ptr.end() - 1);
  for (int s = 0; s < n_faces; ++s) {
    cf[fill[fcell[2 * s]]++] = s << 1;
    if (fcell[2 * s + 1] >= 0) cf[fill[fcell[2 * s + 1]]++] = (s << 1) | 1;
  }
  std::lock_guard<std::mutex> lk(m->mu);
  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  for (void* p : {(void*)m->d_face_cell, (void*)m->d_face_pos, (void*)m->d_cf_ptr,
                  (void*)m->d_cf})
    if (p) cudaFree(p);
  m->d_face_cell = m->d_face_pos = m->d_cf_ptr = m->d_cf = nullptr;
  m->n_faces = 0;
  int st = tf_dev_alloc_bytes(ctx, (void**)&m->d_face_cell, fcell.size() * sizeof(int));
  if (st == TF_OK) st = tf_dev_alloc_bytes(ctx, (void**)&m->d_face_pos, fpos.size() * sizeof(int));
  if (st == TF_OK) st = tf_dev_alloc_bytes(ctx, (void**)&m->d_cf_ptr, ptr.size() * sizeof(int));
  if (st == TF_OK) st = tf_dev_alloc_bytes(ctx, (void**)&m->d_cf, cf.size() * sizeof(int));
  if (st != TF_OK) return st;
  cudaStream_t s = ctx->stream;
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_face_cell, fcell.data(), fcell.size() * sizeof(int),
                              cudaMemcpyHostToDevice, s));
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_face_pos, fpos.data(), fpos.size() * sizeof(int),
                              cudaMemcpyHostToDevice, s));
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_cf_ptr, ptr.data(), ptr.size() * sizeof(int),
                              cudaMemcpyHostToDevice, s));
  TF_CUDA_TRY(cudaMemcpyAsync(m->d_cf, cf.data(), cf.size() * sizeof(int),
                              cudaMemcpyHostToDevice, s));
  TF_CUDA_TRY(cudaStreamSynchronize(s));
  m->n_faces = n_faces;
  return TF_OK;
  TF_API_END
}

namespace {
int grid_for(tf_matrix_s* m, int items) {
  return std::max(1, std::min(m->ctx->sm_count * 8, (items + 255) / 256));
}
}  // namespace

extern "C" int tf_assemble_pressure(tf_ctx ctx, tf_matrix m, const double* d_fc,
                                    const double* d_fw, const double* d_vm,
                                    const int* d_bnd_open, double* d_val) {
  TF_API_BEGIN
  if (!ctx || !m || m->ctx != ctx || !m->d_cf_ptr || !d_fc || !d_fw || !d_val)
    return TF_ERR_ARG;
  std::lock_guard<std::mutex> lk(m->mu);
  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  TF_CUDA_TRY(cudaMemsetAsync(d_val, 0, (size_t)m->nnz * sizeof(double), s));
  if (m->n_faces > 0)
    k_asm_p_off<<<grid_for(m, m->n_faces), 256, 0, s>>>(m->n_faces, m->d_face_cell,
                                                         m->d_face_pos, d_fc, d_fw, d_vm, d_val);
  k_asm_p_diag<<<grid_for(m, m->nt), 256, 0, s>>>(m->nt, m->d_cf_ptr, m->d_cf, m->d_face_cell,
                                                   m->d_dia, d_fc, d_fw, d_vm, d_bnd_open,
                                                   d_val);
  TF_CUDA_TRY(cudaGetLastError());
  return TF_OK;
  TF_API_END
}

extern "C" int tf_assemble_momentum(tf_ctx ctx, tf_matrix m, const double* d_fc,
                                    const double* d_flux, const int* d_bnd_wall, double vis,
                                    double rho, const double* d_vol, double dt, double* d_val) {
  TF_API_BEGIN
  if (!ctx || !m || m->ctx != ctx || !m->d_cf_ptr || !d_fc || !d_flux || !d_vol || !d_val)
    return TF_ERR_ARG;
  std::lock_guard<std::mutex> lk(m->mu);
  TF_CUDA_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  TF_CUDA_TRY(cudaMemsetAsync(d_val, 0, (size_t)m->nnz * sizeof(double), s));
  if (m->n_faces > 0)
    k_asm_m_off<<<grid_for(m, m->n_faces), 256, 0, s>>>(m->n_faces, m->d_face_cell,
                                                         m->d_face_pos, d_fc, d_flux, vis, rho,
                                                         d_val);
  k_asm_m_diag<<<grid_for(m, m->nt), 256, 0, s>>>(m->nt, m->d_cf_ptr, m->d_cf, m->d_face_cell,
                                                   m->d_dia, d_fc, d_flux, d_bnd_wall, vis, rho,
                                                   d_vol, dt, d_val);
  TF_CUDA_TRY(cudaGetLastError());
  return TF_OK;
  TF_API_END
}
