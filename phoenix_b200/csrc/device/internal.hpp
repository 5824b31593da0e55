// Internals shared by the C ABI's translation units (capi.cu, batch.cu, server.cu): error plumbing, the resident
// snapshot object behind the opaque PhxSnapshot handle, and its device views.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/phoenix_b200.h"
#include "../core/ray.cuh"
#include "../host/render_setup.hpp"
#include "../host/snapshot.hpp"

namespace phx_capi {

// Message of the last failed call on this host thread (phx_last_error).
inline std::string& last_error() {
  thread_local std::string e;
  return e;
}


inline int fail(int code, const std::string& msg) {
  last_error() = msg;
  return code;
}

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string& m) : std::runtime_error(m) {}
};

inline void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
T* dev_upload(const T* host, size_t n, std::vector<void*>& owned) {
  T* d = nullptr;
  ck(cudaMalloc((void**)&d, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
  owned.push_back(d);
  if (n) ck(cudaMemcpy(d, host, n * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy H2D");
  return d;
}

// Launches the per-frequency image reduction (spectrum.cu) of a device-resident result.
void launch_spectrum(const PhxRenderParams& p, const PhxFreqOut* d_res, PhxSpectrum* d_spec, cudaStream_t st);

// Device workspace of the synchronous render entry (grown on demand, reused across calls).
struct Workspace {
  int32_t* jobs = nullptr;
  size_t jobs_cap = 0;
  PhxFreqOut* res = nullptr;
  size_t res_cap = 0;
  unsigned long long* counters = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  ~Workspace() {
    cudaFree(jobs);
    cudaFree(res);
    cudaFree(counters);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  }
};

}  // namespace phx_capi

struct PhxHostSnapshot {
  phx::HostSnapshot h;
  std::vector<const int32_t*> maps;
};

struct PhxSnapshot {
  int device = 0;
  int sms = 0;
  char device_name[256] = {0};
  int32_t nleafs = 0, nlevels = 0, cells = 0;
  int32_t nx[3] = {0, 0, 0}, ng[3] = {0, 0, 0}, fd[3] = {0, 0, 0};
  double a = 0, hslope = 0, gam = 0;
  double x_lo[3] = {0, 0, 0}, x_hi[3] = {0, 0, 0};
  float *lb_f = nullptr, *dxc_f = nullptr, *prim_f = nullptr;
  double *lb_d = nullptr, *dxc_d = nullptr, *prim_d = nullptr;
  int32_t* fmap = nullptr;
  int64_t bytes = 0;
  std::vector<void*> owned;
  phx_capi::Workspace ws;
  double read_s = 0.0, decode_s = 0.0, upload_s = 0.0;  // load timings (read + host decode are in read_s)
  bool gpu_decoded = false;
  cudaStream_t stream = nullptr;
  ~PhxSnapshot() {
    if (stream) cudaStreamDestroy(stream);
    for (void* p : owned) cudaFree(p);
  }
};

namespace phx_capi {

template <class R, class PT>
phx::SnapView<R, PT> snap_view(const PhxSnapshot* s, const R* lb, const R* dxc, const PT* prim) {
  phx::SnapView<R, PT> v;
  v.lb = lb;
  v.dxc = dxc;
  v.prim = prim;
  v.fmap = s->fmap;
  for (int d = 0; d < 3; d++) {
    v.fd[d] = s->fd[d];
    v.nx[d] = s->nx[d];
    v.x_lo[1 + d] = R(s->x_lo[d]);
    v.x_hi[1 + d] = R(s->x_hi[d]);
    v.w0[d] = R((s->x_hi[d] - s->x_lo[d]) / s->ng[d]);
    v.iw0up[d] = R(double(1 << (s->nlevels - 1)) * s->ng[d] / (s->x_hi[d] - s->x_lo[d]));
  }
  v.x_lo[0] = v.x_hi[0] = R(0);
  v.nleafs = s->nleafs;
  v.nlevels = s->nlevels;
  v.cells = s->cells;
  v.a = R(s->a);
  v.hs = R(s->hslope);
  v.gam = R(s->gam);
  v.lbd = s->lb_d;
  v.dxcd = s->dxc_d;
  v.a_d = s->a;
  v.hs_d = s->hslope;
  for (int d = 0; d < 3; d++) {
    v.xlo_d[1 + d] = s->x_lo[d];
    v.xhi_d[1 + d] = s->x_hi[d];
    v.w0_d[d] = (s->x_hi[d] - s->x_lo[d]) / s->ng[d];
  }
  v.xlo_d[0] = v.xhi_d[0] = 0.0;
  return v;
}

// The device view of a snapshot for precision mode M with primitives of type PT (FP32 leaf geometry and primitives
// for the FP32 kernels, FP64 geometry for the FP64 kernels; FP64 primitives when PT is double).
template <phx::Mode M, class PT>
phx::SnapView<typename phx::Policy<M>::R, PT> view_for(const PhxSnapshot* s) {
  using R = typename phx::Policy<M>::R;
  const PT* prim;
  if constexpr (sizeof(PT) == 8) prim = s->prim_d; else prim = s->prim_f;
  if constexpr (sizeof(R) == 8) return snap_view<R, PT>(s, s->lb_d, s->dxc_d, prim);
  else return snap_view<R, PT>(s, s->lb_f, s->dxc_f, prim);
}

template <class F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const CudaError& e) {
    return fail(PHX_E_CUDA, e.what());
  } catch (const std::invalid_argument& e) {
    return fail(PHX_E_INVALID, e.what());
  } catch (const std::bad_alloc&) {
    return fail(PHX_E_INVALID, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(PHX_E_IO, e.what());
  }
}

// GPU decode of a dump into s's allocated primitive pool (decode.cu); returns seconds.
double gpu_decode(PhxSnapshot* s, const std::string& dump, const phx::HostSnapshot& meta, int bpol);

}  // namespace phx_capi
