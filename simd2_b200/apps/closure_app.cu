// simd2_closure_app -- drop-in driver for the reference's closure apps
// (apps/{apsp,aplp,mcp,maxrp,minrp,mst,gtc}/{cuASR,emulation}), running the real
// semiring closure on libsimd2.
//
//   simd2_closure_app <app> -f [file] [--bf] [--repeat R] [--out result.bin]
//   simd2_closure_app <app> V density max_weight [--bf] [--repeat R] [--out result.bin]
//   simd2_closure_app gtc V density [--repeat R] [--out result.bin]
//
// Input, as the reference apps read it:
//   -f        "V E" then E lines "u v w" on stdin (mst: a PBBS WeightedEdgeArray
//             file named after -f, symmetric, vertices 0..max id), or
//   V d w     a generated graph: rgg_1d semantics (undirected; per pair i < j
//             one rand() weight in [0, w) then one rand() draw for the edge test
//             `< d`), srand(7); gtc uses the directed variant
//             (apps/data/graph_gen.h:33-81).
// Per-app semiring and fill conventions:
//   apsp  min_plus  non-edge FLT_MAX, diagonal 0, |old-new| > 1e-4 change test
//   aplp  max_plus  non-edge -FLT_MAX, weights truncated to int, APLP change test
//   mcp   max_min   non-edge and diagonal -FLT_MAX
//   maxrp max_mul   non-edge 0
//   minrp min_mul   non-edge FLT_MAX
//   mst   min_max   non-edge FLT_MAX, diagonal 0
//   gtc   or_and    0/1 bytes, diagonal 1
// --bf runs the Bellman-Ford form X <- X (+) A0 (x) X (the reference's APBF build).
// Output line (what scripts/run_apps.py parses): "<avg ms over R runs> <iterations>".
// The time covers the closure on the device (inputs already resident), as the
// reference apps time their loop.
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "simd2.h"

namespace {

struct AppSpec {
  const char* name;
  simd2_op op;
  float fill;
  bool diag_set;
  float diag;
  simd2_conv conv;
  bool int_weights;
};

const AppSpec kApps[] = {
    {"apsp", SIMD2_MIN_PLUS, FLT_MAX, true, 0.0f, SIMD2_CONV_TOL, false},
    {"aplp", SIMD2_MAX_PLUS, -FLT_MAX, false, 0.0f, SIMD2_CONV_APLP, true},
    {"mcp", SIMD2_MAX_MIN, -FLT_MAX, true, -FLT_MAX, SIMD2_CONV_TOL, false},
    {"maxrp", SIMD2_MAX_MUL, 0.0f, false, 0.0f, SIMD2_CONV_TOL, false},
    {"minrp", SIMD2_MIN_MUL, FLT_MAX, false, 0.0f, SIMD2_CONV_TOL, false},
    {"mst", SIMD2_MIN_MAX, FLT_MAX, true, 0.0f, SIMD2_CONV_TOL, false},
    {"gtc", SIMD2_OR_AND, 0.0f, true, 1.0f, SIMD2_CONV_EXACT, false},
};

int usage() {
  fprintf(stderr, "usage: simd2_closure_app <apsp|aplp|mcp|maxrp|minrp|mst|gtc> (-f [file] | V density weight) "
                  "[--bf] [--repeat R] [--out file]\n");
  return 2;
}

// Generated graph with the rgg_1d / rgg_1d_directed draw order.
void generate(std::vector<float>& g, int v, float density, float w, bool directed, float fill) {
  srand(7);
  for (int i = 0; i < v; i++)
    for (int j = 0; j < v; j++) {
      if (i == j) {
        g[(size_t)i * v + j] = 0.0f;
        continue;
      }
      if (directed || j > i) {
        const float weight = (float)rand() / (float)(RAND_MAX / w);
        const float has_edge = (float)rand() / (float)(RAND_MAX / 1);
        const float x = has_edge < density ? weight : fill;
        g[(size_t)i * v + j] = x;
        if (!directed) g[(size_t)j * v + i] = x;
      }
    }
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) return usage();
  const AppSpec* app = nullptr;
  for (const auto& a : kApps)
    if (!strcmp(argv[1], a.name)) app = &a;
  if (!app) return usage();
  bool bf = false;
  int repeat = 10;
  const char* out_path = nullptr;
  std::vector<const char*> pos;
  for (int i = 2; i < argc; i++) {
    if (!strcmp(argv[i], "--bf")) bf = true;
    else if (!strcmp(argv[i], "--repeat") && i + 1 < argc) repeat = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--out") && i + 1 < argc) out_path = argv[++i];
    else pos.push_back(argv[i]);
  }
  if (pos.empty()) return usage();

  int v = 0;
  std::vector<float> g;
  if (!strcmp(pos[0], "-f")) {
    if (!strcmp(app->name, "mst")) {
      if (pos.size() < 2) return usage();
      // PBBS WeightedEdgeArray: header line, then "a b w"; vertices 0..max id
      std::ifstream in(pos[1]);
      std::string line;
      std::getline(in, line);
      std::vector<int> ea, eb;
      std::vector<float> ew;
      int vmax = 0;
      while (std::getline(in, line)) {
        std::istringstream iss(line);
        int a, b;
        float w;
        if (!(iss >> a >> b >> w)) break;
        ea.push_back(a);
        eb.push_back(b);
        ew.push_back(w);
        vmax = std::max(vmax, std::max(a, b));
      }
      v = vmax + 1;
      g.assign((size_t)v * v, 0.0f);
      for (size_t e = 0; e < ea.size(); e++) g[(size_t)ea[e] * v + eb[e]] = g[(size_t)eb[e] * v + ea[e]] = ew[e];
      for (int i = 0; i < v; i++)
        for (int j = 0; j < v; j++)
          if (i != j && g[(size_t)i * v + j] == 0.0f) g[(size_t)i * v + j] = FLT_MAX;
    } else {
      int e = 0;
      if (!(std::cin >> v >> e) || v < 0) return 3;
      g.assign((size_t)v * v, app->fill);
      for (int i = 0; i < e; i++) {
        int a, b;
        float w;
        if (!(std::cin >> a >> b >> w)) return 3;
        if (a < 0 || b < 0 || a >= v || b >= v) return 3;
        g[(size_t)a * v + b] = app->int_weights ? (float)(int)w : w;
      }
      if (app->diag_set)
        for (int i = 0; i < v; i++) g[(size_t)i * v + i] = app->diag;
    }
  } else {
    // gtc takes "V density" (weights fixed at 10, apps/gtc/cuASR/gtc_cuASR.cu), the others "V density weight"
    const bool is_gtc = !strcmp(app->name, "gtc");
    if (pos.size() < (is_gtc ? 2u : 3u)) return usage();
    v = atoi(pos[0]);
    const float density = (float)atof(pos[1]);
    const float w = pos.size() >= 3 ? (float)atof(pos[2]) : 10.0f;
    if (v <= 0 || density < 0 || density > 1) return usage();
    g.assign((size_t)v * v, app->fill);
    const bool directed = !strcmp(app->name, "gtc");
    generate(g, v, density, w, directed, directed ? FLT_MAX : app->fill);
    if (app->diag_set && strcmp(app->name, "gtc"))
      for (int i = 0; i < v; i++) g[(size_t)i * v + i] = app->diag;
  }

  const size_t nn = (size_t)v * v;
  double total_ms = 0.0;
  int iters = 0;
  std::vector<float> result(nn);
  if (app->op == SIMD2_OR_AND) {
    std::vector<uint8_t> t(nn);
    for (size_t x = 0; x < nn; x++) t[x] = (g[x] < FLT_MAX - 100.0f) ? 1 : 0;  // apps/gtc: edge or diagonal
    uint8_t* d = nullptr;
    if (cudaMalloc(&d, std::max(nn, (size_t)1)) != cudaSuccess) return 4;
    for (int r = 0; r < repeat; r++) {
      cudaMemcpy(d, t.data(), nn, cudaMemcpyHostToDevice);
      cudaDeviceSynchronize();
      auto t0 = std::chrono::high_resolution_clock::now();
      int rc = simd2_closure_orand_u8(v, d, v, 500, &iters, nullptr);
      auto t1 = std::chrono::high_resolution_clock::now();
      if (rc && rc != SIMD2_ERR_NOT_CONVERGED) return 10 + rc;
      total_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
    }
    std::vector<uint8_t> r8(nn);
    cudaMemcpy(r8.data(), d, nn, cudaMemcpyDeviceToHost);
    for (size_t x = 0; x < nn; x++) result[x] = r8[x];
    cudaFree(d);
  } else {
    float *d = nullptr, *a0 = nullptr;
    if (cudaMalloc(&d, std::max(nn, (size_t)1) * 4) != cudaSuccess) return 4;
    if (bf && cudaMalloc(&a0, std::max(nn, (size_t)1) * 4) != cudaSuccess) return 4;
    if (bf) cudaMemcpy(a0, g.data(), nn * 4, cudaMemcpyHostToDevice);
    for (int r = 0; r < repeat; r++) {
      cudaMemcpy(d, g.data(), nn * 4, cudaMemcpyHostToDevice);
      cudaDeviceSynchronize();
      auto t0 = std::chrono::high_resolution_clock::now();
      int rc = bf ? simd2_closure_bf(app->op, v, a0, v, d, v, 500, app->conv, &iters, nullptr)
                  : simd2_closure(app->op, v, d, v, 500, app->conv, &iters, nullptr);
      auto t1 = std::chrono::high_resolution_clock::now();
      if (rc && rc != SIMD2_ERR_NOT_CONVERGED) return 10 + rc;
      total_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
    }
    cudaMemcpy(result.data(), d, nn * 4, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (a0) cudaFree(a0);
  }
  if (out_path) {
    FILE* f = fopen(out_path, "wb");
    if (!f) return 5;
    fwrite(&v, 4, 1, f);
    fwrite(result.data(), 4, nn, f);
    fclose(f);
  }
  printf("%f %d\n", total_ms / repeat, iters);
  return 0;
}
