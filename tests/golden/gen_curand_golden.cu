// Fixture generator: records what the CUDA toolkit's cuRAND device API returns
// for the Philox4_32_10 generator, so that the oracle's own Philox restatement
// (oracle/sa_oracle.cpp) can be pinned against it without a GPU.
//
// The reference seeds one Philox state per lattice site with
// curand_init(seed, site, 0, &state) (src/random.cu:15-23), draws the coupling
// words with curand() (src/random.cu:25-35) and one curand_uniform() per site
// per half-sweep (src/device_2d.cu:96-97, src/device_3d.cu:43-44). This program
// only CALLS those library functions and writes their results to JSON.
//
// Build + run (needs a GPU):
//   nvcc -gencode arch=compute_100a,code=sm_100a -O2 -o gen_curand_golden \
//        tests/golden/gen_curand_golden.cu
//   ./gen_curand_golden > tests/golden/curand_philox_golden.json
//   ./gen_curand_golden --bulk curand_bulk.bin
//   python tests/golden/hash_curand_bulk.py curand_bulk.bin > tests/golden/curand_philox_bulk.json
// --bulk writes, for each seed of kBulkSeeds, the first kBulkDraws curand()
// outputs and the first kBulkDraws curand_uniform() bit patterns of every
// subsequence 0..kBulkSubs-1 (offset 0), as little-endian u32:
// [seed][u32 | uniform][subsequence][draw].
#include <cstdio>
#include <cstring>
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>
#include <curand_kernel.h>

struct Case {
  unsigned long long seed, subseq, offset;
};

constexpr int kDraws = 20;
constexpr int kBulkSubs = 4096, kBulkDraws = 64;
const unsigned long long kBulkSeeds[] = {1ULL, 2ULL, 3ULL, 4ULL, 1234ULL, 1000ULL, 1001ULL, 1002ULL, 1003ULL};

__global__ void bulk_kernel(unsigned long long seed, unsigned* u32_out, unsigned* uni_out) {
  int sub = blockIdx.x * blockDim.x + threadIdx.x;
  if (sub >= kBulkSubs) return;
  curandStatePhilox4_32_10_t a, b;
  curand_init(seed, (unsigned long long)sub, 0ULL, &a);
  curand_init(seed, (unsigned long long)sub, 0ULL, &b);
  for (int k = 0; k < kBulkDraws; ++k) {
    u32_out[sub * kBulkDraws + k] = curand(&a);
    const float f = curand_uniform(&b);
    unsigned bits;
    memcpy(&bits, &f, 4);
    uni_out[sub * kBulkDraws + k] = bits;
  }
}

__global__ void draw_kernel(const Case* cases, int n, unsigned* u32_out,
                            float* uni_out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  curandStatePhilox4_32_10_t a, b;
  curand_init(cases[i].seed, cases[i].subseq, cases[i].offset, &a);
  curand_init(cases[i].seed, cases[i].subseq, cases[i].offset, &b);
  for (int k = 0; k < kDraws; ++k) {
    u32_out[i * kDraws + k] = curand(&a);
    uni_out[i * kDraws + k] = curand_uniform(&b);
  }
}

#define CK(x)                                                              \
  do {                                                                     \
    cudaError_t e = (x);                                                   \
    if (e != cudaSuccess) {                                                \
      fprintf(stderr, "%s:%d %s\n", __FILE__, __LINE__, cudaGetErrorString(e)); \
      return 1;                                                            \
    }                                                                      \
  } while (0)

static int bulk(const char* path) {
  const size_t per = (size_t)kBulkSubs * kBulkDraws;
  unsigned *d_u, *d_f;
  CK(cudaMalloc(&d_u, per * sizeof(unsigned)));
  CK(cudaMalloc(&d_f, per * sizeof(unsigned)));
  FILE* out = fopen(path, "wb");
  if (!out) {
    fprintf(stderr, "cannot open %s\n", path);
    return 1;
  }
  std::vector<unsigned> h(per);
  for (unsigned long long seed : kBulkSeeds) {
    bulk_kernel<<<kBulkSubs / 128, 128>>>(seed, d_u, d_f);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    CK(cudaMemcpy(h.data(), d_u, per * sizeof(unsigned), cudaMemcpyDeviceToHost));
    fwrite(h.data(), sizeof(unsigned), per, out);
    CK(cudaMemcpy(h.data(), d_f, per * sizeof(unsigned), cudaMemcpyDeviceToHost));
    fwrite(h.data(), sizeof(unsigned), per, out);
  }
  fclose(out);
  cudaFree(d_u);
  cudaFree(d_f);
  return 0;
}

int main(int argc, char** argv) {
  if (argc == 3 && strcmp(argv[1], "--bulk") == 0) return bulk(argv[2]);
  std::vector<Case> cases;
  const unsigned long long seeds[] = {0ULL, 1ULL, 2ULL, 3ULL, 4ULL, 1234ULL,
                                      1000ULL, 1001ULL, 1002ULL, 1003ULL,
                                      0xDEADBEEFCAFEF00DULL};
  const unsigned long long subs[] = {0ULL, 1ULL, 2ULL, 3ULL, 63ULL, 4095ULL,
                                     4096ULL, 32767ULL, 262143ULL,
                                     (1ULL << 32) | 5ULL, (1ULL << 40) + 3ULL};
  for (unsigned long long s : seeds)
    for (unsigned long long q : subs) cases.push_back({s, q, 0ULL});
  const unsigned long long offs[] = {1ULL, 2ULL, 3ULL, 4ULL, 5ULL, 6ULL, 7ULL,
                                     13ULL, 1000001ULL, (1ULL << 32) + 3ULL,
                                     (1ULL << 34) + 2ULL};
  for (unsigned long long o : offs) cases.push_back({7ULL, 11ULL, o});
  for (unsigned long long o : offs) cases.push_back({1234ULL, 4095ULL, o});

  int n = (int)cases.size();
  Case* d_cases;
  unsigned* d_u;
  float* d_f;
  CK(cudaMalloc(&d_cases, n * sizeof(Case)));
  CK(cudaMalloc(&d_u, n * kDraws * sizeof(unsigned)));
  CK(cudaMalloc(&d_f, n * kDraws * sizeof(float)));
  CK(cudaMemcpy(d_cases, cases.data(), n * sizeof(Case), cudaMemcpyHostToDevice));
  draw_kernel<<<(n + 127) / 128, 128>>>(d_cases, n, d_u, d_f);
  CK(cudaGetLastError());
  CK(cudaDeviceSynchronize());
  std::vector<unsigned> u(n * kDraws);
  std::vector<float> f(n * kDraws);
  CK(cudaMemcpy(u.data(), d_u, u.size() * sizeof(unsigned), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(f.data(), d_f, f.size() * sizeof(float), cudaMemcpyDeviceToHost));

  printf("{\n  \"generator\": \"curand Philox4_32_10 device API (curand_init/curand/curand_uniform)\",\n");
  printf("  \"draws_per_case\": %d,\n  \"cases\": [\n", kDraws);
  for (int i = 0; i < n; ++i) {
    printf("    {\"seed\": \"%llu\", \"subsequence\": \"%llu\", \"offset\": \"%llu\",\n",
           cases[i].seed, cases[i].subseq, cases[i].offset);
    printf("     \"u32\": [");
    for (int k = 0; k < kDraws; ++k)
      printf("%s%u", k ? ", " : "", u[i * kDraws + k]);
    printf("],\n     \"uniform_bits\": [");
    for (int k = 0; k < kDraws; ++k) {
      unsigned bits;
      memcpy(&bits, &f[i * kDraws + k], 4);
      printf("%s%u", k ? ", " : "", bits);
    }
    printf("]}%s\n", i + 1 < n ? "," : "");
  }
  printf("  ]\n}\n");
  cudaFree(d_cases);
  cudaFree(d_u);
  cudaFree(d_f);
  return 0;
}
