// ref_harness.cpp -- HDF5-free driver for the reference's own hypJacL2,
// linked with the reference sources built for sm_100a (oracle/Makefile).
//
// TEST INFRASTRUCTURE ONLY: it runs the reference as the parity checker (the
// golden fixtures in tests/golden/ are its outputs).  It mirrors the
// argument handling of the reference CLI 1/main.cu:10-160 without HDF5:
//
//   ref_harness DEV SDY SNP0 SNP1 ALG NPLUS M N IN.bin OUT.bin [REPS]
//
// REPS (default 1) runs hypJacL2 that many times on the same input (G
// restored before each run) and prints one line per run to stdout,
// "REP r ret sweeps wall setup compute cleanup" (the reference's timing[4],
// seconds); OUT.bin holds the last run.
// IN.bin : M*N doubles, Fortran order, LDA = M.
// OUT.bin: int32 ret, uint32 sweeps, uint64 rot_s, uint64 rot_b,
//          double timing[4], double G[M*N], double V[N*N] (ALG & 2), double D[N].
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

extern "C" int configureGPU(const int dev) throw();
extern "C" void init_strats(const char *const sdy, const char *const snp0, const unsigned n0,
                            const char *const snp1, const unsigned n1) throw();
extern "C" int hypJacL2(const unsigned routine, const unsigned nrow, const unsigned ncol,
                        const unsigned nplus, double *const hG, const unsigned ldhG, double *const hV,
                        const unsigned ldhV, double *const hD, unsigned *const glbSwp,
                        unsigned long long *const glb_s, unsigned long long *const glb_b,
                        double *const timing) throw();

int main(int argc, char **argv)
{
  if (argc != 11 && argc != 12) {
    std::fprintf(stderr, "%s DEV SDY SNP0 SNP1 ALG NPLUS M N IN.bin OUT.bin [REPS]\n", argv[0]);
    return EXIT_FAILURE;
  }
  const int dev = std::atoi(argv[1]);
  const unsigned alg = (unsigned)std::atoi(argv[5]);
  const unsigned nplus = (unsigned)std::atoi(argv[6]);
  const unsigned m = (unsigned)std::atoi(argv[7]);
  const unsigned n = (unsigned)std::atoi(argv[8]);
  const int reps = (argc == 12) ? std::atoi(argv[11]) : 1;
  if (reps < 1)
    return EXIT_FAILURE;

  init_strats(argv[2], argv[3], 32u, argv[4], (n + 15u) / 16u);
  if (configureGPU(dev) < 30)
    return EXIT_FAILURE;

  double *hG = nullptr, *hV = nullptr, *hD = nullptr;
  if (cudaHostAlloc((void **)&hG, sizeof(double) * m * n, cudaHostAllocPortable) != cudaSuccess)
    return EXIT_FAILURE;
  if ((alg & 2u) && cudaHostAlloc((void **)&hV, sizeof(double) * m * n, cudaHostAllocPortable) != cudaSuccess)
    return EXIT_FAILURE;
  if (cudaHostAlloc((void **)&hD, sizeof(double) * n, cudaHostAllocPortable) != cudaSuccess)
    return EXIT_FAILURE;

  FILE *f = std::fopen(argv[9], "rb");
  if (!f || std::fread(hG, sizeof(double), (size_t)m * n, f) != (size_t)m * n)
    return EXIT_FAILURE;
  std::fclose(f);
  std::vector<double> g0;
  if (reps > 1)
    g0.assign(hG, hG + (size_t)m * n);

  unsigned swp = 0u;
  unsigned long long s = 0ull, b = 0ull;
  double timing[4] = {0.0, 0.0, 0.0, 0.0};
  int ret = 0;
  for (int r = 0; r < reps; ++r) {
    if (r)
      std::memcpy(hG, g0.data(), sizeof(double) * g0.size());
    // as 1/main.cu:78-80: V is allocated with the leading dimension of G
    ret = hypJacL2(alg, m, n, nplus, hG, m, hV, (alg & 2u) ? m : 0u, hD, &swp, &s, &b, timing);
    if (reps > 1)
      std::printf("REP %d %d %u %.9f %.9f %.9f %.9f\n", r, ret, swp, timing[0], timing[1], timing[2], timing[3]);
  }

  f = std::fopen(argv[10], "wb");
  if (!f)
    return EXIT_FAILURE;
  const int r32 = ret;
  std::fwrite(&r32, sizeof(r32), 1, f);
  std::fwrite(&swp, sizeof(swp), 1, f);
  std::fwrite(&s, sizeof(s), 1, f);
  std::fwrite(&b, sizeof(b), 1, f);
  std::fwrite(timing, sizeof(double), 4, f);
  std::fwrite(hG, sizeof(double), (size_t)m * n, f);
  if (alg & 2u) // only the first N rows of each column of V are written by hypJacL2
    for (unsigned c = 0u; c < n; ++c)
      std::fwrite(hV + (size_t)c * m, sizeof(double), n, f);
  std::fwrite(hD, sizeof(double), n, f);
  std::fclose(f);

  cudaFreeHost(hD);
  if (hV)
    cudaFreeHost(hV);
  cudaFreeHost(hG);
  cudaDeviceReset();
  return 0;
}
