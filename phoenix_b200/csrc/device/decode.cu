// GPU decode of a BHAC dump: conserved -> primitive on the device, streamed from the file in leaf chunks.
//
// The reference's gpu_decode path (src/device/kernel.cu:105-112 k_decode, 200-260 decode_to_device) reads the dump
// in chunks into pinned memory, copies each chunk to the device and decodes it there while the host reads the next
// one.  Here the same pipeline runs on two pinned/device buffer pairs and two streams: the host reads chunk k+1 while
// chunk k is copied and decoded, and each cell is decoded by one thread with the same FP64 routine the host reader
// uses (core/decode.cuh: metric at the Simpson-weighted centroid, convert2prim of bhac.hpp:247-346).  The primitives
// land directly in the snapshot's device pool (FP32, and FP64 when the snapshot keeps it).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <string>

#include "../core/decode.cuh"
#include "internal.hpp"

namespace phx {

struct DecodeArgs {
  const double* cons;  // nl leaf blocks, each nwini arrays of `cells` doubles
  const double* lb;    // [nleafs][3] device FP64 leaf origins
  const double* dxc;   // [nleafs][3] device FP64 cell sizes
  float* prim_f;       // [nleafs][cells][8]
  double* prim_d;      // same in FP64, or null
  double a, hs, gam;
  int32_t bpol, nwini, cells, l0, nl;
  int32_t nx[3];
};

__global__ void __launch_bounds__(128) k_decode(const __grid_constant__ DecodeArgs A) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)A.nl * A.cells) return;
  const int q = (int)(t / A.cells), cell = (int)(t - (long long)q * A.cells);
  const size_t l = (size_t)A.l0 + q;
  const double lb3[3] = {A.lb[3 * l], A.lb[3 * l + 1], A.lb[3 * l + 2]};
  const double dx3[3] = {A.dxc[3 * l], A.dxc[3 * l + 1], A.dxc[3 * l + 2]};
  double p[kNPrim];
  cons_to_prim(A.a, A.hs, A.gam, A.bpol, A.nwini, A.nx, lb3, dx3, A.cons + (size_t)q * A.nwini * A.cells, cell, p);
  const size_t o = (l * A.cells + cell) * kNPrim;
  float4* pf = reinterpret_cast<float4*>(A.prim_f + o);
  pf[0] = make_float4((float)p[0], (float)p[1], (float)p[2], (float)p[3]);
  pf[1] = make_float4((float)p[4], (float)p[5], (float)p[6], (float)p[7]);
  if (A.prim_d)
    for (int v = 0; v < kNPrim; v++) A.prim_d[o + v] = p[v];
}

}  // namespace phx

namespace phx_capi {

// Decodes the dump's cells into s's device primitive pool (allocated, not yet filled); returns the seconds spent.
double gpu_decode(PhxSnapshot* s, const std::string& dump, const phx::HostSnapshot& meta, int bpol) {
  const auto t0 = std::chrono::steady_clock::now();
  const size_t leaf_doubles = (size_t)meta.nwini * meta.cells;
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>(meta.nleafs, (64u << 20) / (leaf_doubles * 8)));
  double* host[2] = {nullptr, nullptr};
  double* dev[2] = {nullptr, nullptr};
  cudaStream_t st[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  auto release = [&]() {
    for (int b = 0; b < 2; b++) {
      if (st[b]) cudaStreamSynchronize(st[b]);
      if (done[b]) cudaEventDestroy(done[b]);
      if (st[b]) cudaStreamDestroy(st[b]);
      cudaFreeHost(host[b]);
      cudaFree(dev[b]);
    }
  };
  try {
    for (int b = 0; b < 2; b++) {
      ck(cudaHostAlloc((void**)&host[b], (size_t)chunk * leaf_doubles * sizeof(double), cudaHostAllocDefault),
         "cudaHostAlloc decode buffer");
      ck(cudaMalloc((void**)&dev[b], (size_t)chunk * leaf_doubles * sizeof(double)), "cudaMalloc decode buffer");
      ck(cudaStreamCreateWithFlags(&st[b], cudaStreamNonBlocking), "cudaStreamCreate");
      ck(cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming), "cudaEventCreate");
      ck(cudaEventRecord(done[b], st[b]), "event");
    }
    phx::DecodeArgs A;
    A.lb = s->lb_d;
    A.dxc = s->dxc_d;
    A.prim_f = s->prim_f;
    A.prim_d = s->prim_d;
    A.a = meta.a;
    A.hs = meta.hslope;
    A.gam = meta.gam;
    A.bpol = bpol;
    A.nwini = meta.nwini;
    A.cells = meta.cells;
    for (int d = 0; d < 3; d++) A.nx[d] = meta.nx[d];
    int cur = 0;
    phx::stream_leaf_blocks(
        dump, meta, chunk,
        [&](int l0, int) {
          cur = (l0 / chunk) & 1;
          ck(cudaEventSynchronize(done[cur]), "decode buffer");  // its previous chunk has been copied and decoded
          return host[cur];
        },
        [&](int l0, int nl, const double* buf) {
          ck(cudaMemcpyAsync(dev[cur], buf, (size_t)nl * leaf_doubles * sizeof(double), cudaMemcpyHostToDevice,
                             st[cur]),
             "H2D conserved chunk");
          phx::DecodeArgs a = A;
          a.cons = dev[cur];
          a.l0 = l0;
          a.nl = nl;
          const long long n = (long long)nl * meta.cells;
          phx::k_decode<<<(unsigned)((n + 127) / 128), 128, 0, st[cur]>>>(a);
          ck(cudaGetLastError(), "decode launch");
          ck(cudaEventRecord(done[cur], st[cur]), "event");
        });
    for (int b = 0; b < 2; b++) ck(cudaStreamSynchronize(st[b]), "decode");
  } catch (...) {
    release();
    throw;
  }
  release();
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace phx_capi
