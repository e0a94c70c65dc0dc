// A PLD-style caller: the data flow of apps/pld/cuASR/test.cpp around
// knn_mxu (reference points stored [dim][ref_nb] and transposed on the host
// to [ref_nb][dim], queries [dim][query_nb], results [k][query_nb]), built
// against simd2_cuasr.h.  Reads ref_nb, query_nb, dim, k and the two point
// arrays from argv[1]; writes the distances then the indices to argv[2].
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "simd2.h"
#include "simd2_cuasr.h"

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 3;
  int hdr[4];
  if (fread(hdr, sizeof(int), 4, f) != 4) return 4;
  const int ref_nb = hdr[0], query_nb = hdr[1], dim = hdr[2], k = hdr[3];
  std::vector<float> ref((size_t)ref_nb * dim), query((size_t)query_nb * dim);
  if (fread(ref.data(), sizeof(float), ref.size(), f) != ref.size()) return 5;
  if (fread(query.data(), sizeof(float), query.size(), f) != query.size()) return 6;
  fclose(f);
  std::vector<float> ref_t(ref.size());
  for (int i = 0; i < ref_nb; i++)
    for (int j = 0; j < dim; j++) ref_t[(size_t)i * dim + j] = ref[(size_t)j * ref_nb + i];
  std::vector<float> dist((size_t)query_nb * k);
  std::vector<int> index((size_t)query_nb * k);
  double t = 0.0;
  if (!knn_mxu(ref_t.data(), ref_nb, query.data(), query_nb, dim, k, dist.data(), index.data(), &t)) return 7;
  if (!(t > 0.0)) return 8;
  FILE* o = fopen(argv[2], "wb");
  if (!o) return 9;
  fwrite(dist.data(), sizeof(float), dist.size(), o);
  fwrite(index.data(), sizeof(int), index.size(), o);
  fclose(o);
  return 0;
}
