// A closure app written against the reference's own interface: the loop of
// apps/apsp/cuASR/apsp_cuASR.cu:42-54 (cuasr_minplus_srsgemm + comp_update),
// the swapped row-major call of tests/cuAsr_kernel_test.cu:60 and
// tensor_srgemm, compiled against include/simd2_cuasr.h and libsimd2.
//
//   cuasr_app <in.bin> <out.bin>
// in.bin : int32 v, then v*v float32 adjacency (row-major)
// out.bin: int32 iterations, v*v float32 closure, then the row-major
//          one-shot products (swapped cuASR call, tensor_srgemm) of the
//          16 x 16 top-left block with itself, 2 x 256 float32.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "simd2_cuasr.h"

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 3;
  int v = 0;
  if (fread(&v, 4, 1, f) != 1) return 4;
  std::vector<float> adj((size_t)v * v);
  if (fread(adj.data(), 4, adj.size(), f) != adj.size()) return 5;
  fclose(f);

  float *out_d, *out_d_delta;
  int* check_d;
  int check_h[1];
  cudaMalloc(&check_d, sizeof(int));
  cudaMalloc(&out_d, adj.size() * 4);
  cudaMalloc(&out_d_delta, adj.size() * 4);
  cudaMemcpy(out_d, adj.data(), adj.size() * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(out_d_delta, adj.data(), adj.size() * 4, cudaMemcpyHostToDevice);
  bool run = true;
  int num_itr = 0;
  while (run && num_itr < 500) {
    num_itr += 1;
    int retval = cuasr_minplus_srsgemm(v, v, v, out_d, v, out_d, v, out_d, v, out_d_delta, true, nullptr);
    if (retval) return 10;
    cudaDeviceSynchronize();
    run = comp_update(out_d, out_d_delta, check_d, check_h, v, v);
  }
  std::vector<float> dist(adj.size());
  cudaMemcpy(dist.data(), out_d, adj.size() * 4, cudaMemcpyDeviceToHost);

  // one-shot 16 x 16 products of the adjacency's top-left block
  const int m = 16;
  std::vector<float> a(m * m);
  std::vector<half> ah(m * m);
  for (int i = 0; i < m; i++)
    for (int j = 0; j < m; j++) {
      float x = adj[(size_t)i * v + j];
      a[i * m + j] = x > 1e30f ? 60000.f : x;  // keep it finite in half
      ah[i * m + j] = __float2half(a[i * m + j]);
    }
  float *da, *dc, *dd1, *dd2;
  half* dh;
  cudaMalloc(&da, m * m * 4);
  cudaMalloc(&dc, m * m * 4);
  cudaMalloc(&dd1, m * m * 4);
  cudaMalloc(&dd2, m * m * 4);
  cudaMalloc(&dh, m * m * 2);
  cudaMemcpy(da, a.data(), m * m * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(dh, ah.data(), m * m * 2, cudaMemcpyHostToDevice);
  cudaMemset(dc, 0, m * m * 4);
  // row-major D = A (x) A via the swapped column-major call (N, M, K, B, ldb, A, lda)
  if (cuasr_minplus_srsgemm(m, m, m, da, m, da, m, dc, m, dd1, false, nullptr)) return 11;
  if (tensor_srgemm(dh, dh, dc, dd2, m, m, m, false, min_plus) != 0) return 12;
  if (tensor_srgemm(dh, dh, dc, dd2, 15, m, m, false, min_plus) != -1) return 13;
  cudaDeviceSynchronize();
  std::vector<float> r1(m * m), r2(m * m);
  cudaMemcpy(r1.data(), dd1, m * m * 4, cudaMemcpyDeviceToHost);
  cudaMemcpy(r2.data(), dd2, m * m * 4, cudaMemcpyDeviceToHost);

  FILE* o = fopen(argv[2], "wb");
  fwrite(&num_itr, 4, 1, o);
  fwrite(dist.data(), 4, dist.size(), o);
  fwrite(r1.data(), 4, r1.size(), o);
  fwrite(r2.data(), 4, r2.size(), o);
  fclose(o);
  return cudaGetLastError() == cudaSuccess ? 0 : 20;
}
