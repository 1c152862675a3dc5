// x1.cpp -- the x1 command line over libgjx.so, after the reference's test
// driver 1/main.cu:10-160:
//
//   x1 DEV SDY SNP0 SNP1 ALG H5F H5G [H5R]
//
// DEV: CUDA device; SDY: strategy library (strat.so); SNP0/SNP1: inner and
// outer strategy names; ALG: the hypJacL2 routine bits; H5F/H5G: input file
// and group, holding IDADIM = {LDA, M, N, NPLUS} (int) and G (double,
// N x LDA in C order, i.e. column-major LDA x N); the group's name is N, from
// which the outer table size n1 = ceil(N / 16) is taken, as the reference
// does.  With H5R, the group H5G is created in H5R (the file is created if
// absent) holding IDADIM, ISTATS = {sweeps or error, STRAT0, STRAT1, error},
// TIMING[4], G (U), V (ALG & 2) and D.  Exit status: hypJacL2's return.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "gjx.h"
#include "h5mini.h"

namespace {

[[noreturn]] void die(const std::string &m)
{
  (void)std::fprintf(stderr, "[ERROR] x1: %s\n", m.c_str());
  std::exit(EXIT_FAILURE);
}

bool fexist(const char *p)
{
  struct stat st;
  return p && !stat(p, &st);
}

} // namespace

int main(int argc, char *argv[])
{
  if (argc < 8 || argc > 9) {
    (void)std::fprintf(stderr, "%s DEV SDY SNP0 SNP1 ALG H5F H5G [H5R]\n", argv[0]);
    return EXIT_FAILURE;
  }
  const char *const ca_dev = argv[1], *const ca_sdy = argv[2], *const ca_snp0 = argv[3], *const ca_snp1 = argv[4],
                    *const ca_alg = argv[5], *const ca_h5f = argv[6], *const ca_h5g = argv[7];
  const char *const ca_h5r = (argc == 9) ? argv[8] : nullptr;

  const unsigned n0 = 32u;
  const unsigned n1 = (unsigned)(std::atoi(ca_h5g) + 15) / 16u;
  init_strats(ca_sdy, ca_snp0, n0, ca_snp1, n1); // exits on error, as the reference's

  const int dev = std::atoi(ca_dev);
  const int dcc = gjx_configure_device(dev);
  if (dcc != 100)
    die("device " + std::to_string(dev) + " has compute capability " + std::to_string(dcc) +
        "; this build runs on 10.0 (sm_100a) only");
  gjx_set_verbose(0);

  const unsigned routine = (unsigned)std::atoi(ca_alg);
  if (!fexist(ca_h5f))
    die(std::string("non-existent H5F(") + ca_h5f + ")");

  std::string err;
  h5m::Array a;
  std::vector<int> idadim;
  if (!h5m::read(ca_h5f, std::string(ca_h5g) + "/IDADIM", a, err) || !a.to_int(idadim) || idadim.size() < 4u)
    die("IDADIM: " + (err.empty() ? std::string("not 4 integers") : err));
  const unsigned ldhG = (unsigned)idadim[0], nrow = (unsigned)idadim[1], ncol = (unsigned)idadim[2],
                 nplus = (unsigned)idadim[3];
  if (idadim[0] < 0 || idadim[1] < 0 || idadim[2] < 0 || idadim[3] < 0)
    die("negative entry in IDADIM");

  std::vector<double> hG;
  if (!h5m::read(ca_h5f, std::string(ca_h5g) + "/G", a, err) || !a.to_double(hG))
    die("G: " + err);
  if ((unsigned long long)hG.size() != (unsigned long long)ldhG * ncol)
    die("G holds " + std::to_string(hG.size()) + " values, IDADIM asks for LDA * N = " +
        std::to_string((unsigned long long)ldhG * ncol));

  std::vector<double> hV, hD(ncol ? ncol : 1u);
  unsigned ldhV = 0u;
  if (routine & 2u) {
    hV.assign((size_t)ldhG * ncol, 0.0);
    ldhV = ldhG;
  }

  unsigned glbSwp = 0u;
  unsigned long long glb_s = 0ull, glb_b = 0ull;
  double timing[4] = {-0.0, -0.0, -0.0, -0.0};
  const int ret = hypJacL2(routine, nrow, ncol, nplus, hG.data(), ldhG, hV.empty() ? nullptr : hV.data(), ldhV,
                           hD.data(), &glbSwp, &glb_s, &glb_b, timing);
  if (ret)
    (void)std::fprintf(stderr, "%s: error %d\n", argv[0], ret);
  else {
    (void)std::fprintf(stdout, "GLB_ROT_S(%20llu), GLB_ROT_B(%20llu)\n", glb_s, glb_b);
    (void)std::fflush(stdout);
    (void)std::fprintf(stdout, "%#12.6f s %2u sweeps\n", *timing, glbSwp);
    (void)std::fflush(stdout);
  }

  if (ca_h5r) {
    unsigned s0 = 0u, st0, pr0, s1 = 0u, st1, pr1;
    (void)gjx_strat_info(&s0, &st0, &pr0, &s1, &st1, &pr1);
    const int ida[4] = {(int)ldhG, (int)nrow, (int)ncol, (int)nplus};
    const int istats[4] = {(ret < 0) ? ret : (int)glbSwp, (int)s0, (int)s1, ret};
    std::vector<h5m::NewDataset> ds;
    ds.push_back({"IDADIM", {4u}, false, ida});
    ds.push_back({"ISTATS", {4u}, false, istats});
    ds.push_back({"TIMING", {4u}, true, timing});
    ds.push_back({"G", {ncol, ldhG}, true, hG.data()});
    if (!hV.empty())
      ds.push_back({"V", {ncol, ldhV}, true, hV.data()});
    ds.push_back({"D", {ncol}, true, hD.data()});
    if (!h5m::write_group(ca_h5r, ca_h5g, ds, fexist(ca_h5r) ? 1 : 0, err))
      die("H5R: " + err);
  }
  return ret;
}
