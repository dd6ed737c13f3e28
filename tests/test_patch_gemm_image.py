"""CPU test of the operand image of the tensor-core patch-GEMM smoother
(patch_gemm_image in csrc/fe_data.cpp): a host emulation of the kernel's data
path for one patch -- z-fold of the box into e = u(p) + u(N1-1-p) and
o = u(p) - u(N1-1-p), the GEMMs with the TF32 image decoded through the same
K-major operand layout the kernel's descriptors use, and the unfold
E +- O -- must reproduce the FP64 patch solve x_I = A_II^{-1} (b_I - A_IB x_B)
to TF32 accuracy, with zero padding rows."""
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(REPO, "gputensorproductsmoother_b200", "csrc")

HARNESS = r"""
#include "fe_data.h"
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
using namespace tps;
int main(int argc, char **argv) {
  const int ck = atoi(argv[1]);
  for (int k = 2; k <= 4; ++k) {
    DegreeData D = make_degree_data(k);
    const int n1 = 2*k+1, m = 2*k-1, pl = n1*n1, ipl = m*m, nb = n1*n1*n1, ni = m*m*m;
    const int ke = (k+1)*pl, ko = k*pl, ne = k*ipl, no = (k-1)*ipl;
    const int nbe = (ne+15)/16*16, nbo = (no+15)/16*16, ce = (ke+ck-1)/ck, co = (ko+ck-1)/ck;
    std::vector<float> img = patch_gemm_image(D, nbe, nbo, ck);
    if (img.size() != (size_t)ce*nbe*ck + (size_t)co*nbo*ck) { printf("SIZE %d\n", k); return 1; }
    auto get = [&](const float *base, int n, int kk) {
      return base[((n >> 3) * (ck / 4) * 128 + (n & 7) * 16 + (kk >> 2) * 128 + (kk & 3) * 4) / 4];
    };
    std::mt19937 rng(k); std::uniform_real_distribution<double> U(-1, 1);
    std::vector<double> u(nb); for (auto &v : u) v = U(rng);
    std::vector<double> inv = dense_patch_inverse(D, 3), r(ni), xref(ni, 0.0);
    const double *Mm = D.pmass.data(), *Ll = D.plap.data();
    for (int i = 0; i < ni; ++i) {
      int ix = 1 + i % m, iy = 1 + (i/m) % m, iz = 1 + i/(m*m);
      double acc = u[ix + n1*(iy + n1*iz)];
      for (int q = 0; q < nb; ++q) {
        int qx = q % n1, qy = (q/n1) % n1, qz = q/pl;
        if (!(qx==0||qx==n1-1||qy==0||qy==n1-1||qz==0||qz==n1-1)) continue;
        acc -= (Ll[ix*n1+qx]*Mm[iy*n1+qy]*Mm[iz*n1+qz] + Mm[ix*n1+qx]*Ll[iy*n1+qy]*Mm[iz*n1+qz] +
                Mm[ix*n1+qx]*Mm[iy*n1+qy]*Ll[iz*n1+qz]) * u[q];
      }
      r[i] = acc;
    }
    for (int i = 0; i < ni; ++i) for (int j = 0; j < ni; ++j) xref[i] += inv[(size_t)i*ni+j]*r[j];
    std::vector<double> e(ce*ck, 0.0), o(co*ck, 0.0);
    for (int kq = 0; kq < ke; ++kq) {
      int p = kq / pl, s = kq % pl;
      double u1 = u[p*pl + s], u2 = p < k ? u[(n1-1-p)*pl + s] : 0.0;
      e[kq] = u1 + u2;
      if (kq < ko) o[kq] = u1 - u2;
    }
    std::vector<double> E(nbe, 0.0), O(nbo, 0.0);
    double pad = 0.0;
    for (int c = 0; c < ce; ++c) for (int n = 0; n < nbe; ++n) for (int kk = 0; kk < ck; ++kk) {
      const float g = get(img.data() + (size_t)c*nbe*ck, n, kk);
      E[n] += g * e[c*ck+kk];
      if (n >= ne || c*ck + kk >= ke) pad += std::fabs(g);
    }
    const float *go = img.data() + (size_t)ce*nbe*ck;
    for (int c = 0; c < co; ++c) for (int n = 0; n < nbo; ++n) for (int kk = 0; kk < ck; ++kk) {
      const float g = get(go + (size_t)c*nbo*ck, n, kk);
      O[n] += g * o[c*ck+kk];
      if (n >= no || c*ck + kk >= ko) pad += std::fabs(g);
    }
    double err = 0.0, mx = 0.0;
    for (int zp = 0; zp < k; ++zp) for (int rr = 0; rr < ipl; ++rr) {
      if (zp < k-1) {
        err = std::max(err, std::fabs(E[zp*ipl+rr] + O[zp*ipl+rr] - xref[zp*ipl+rr]));
        err = std::max(err, std::fabs(E[zp*ipl+rr] - O[zp*ipl+rr] - xref[(m-1-zp)*ipl+rr]));
      } else {
        err = std::max(err, std::fabs(E[zp*ipl+rr] - xref[zp*ipl+rr]));
      }
    }
    for (double v : xref) mx = std::max(mx, std::fabs(v));
    printf("%d %.6e %.6e\n", k, err / mx, pad);
  }
  return 0;
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    d = tmp_path_factory.mktemp("pg")
    src = d / "pg.cpp"
    src.write_text(HARNESS)
    exe = d / "pg"
    subprocess.run([gxx, "-O2", "-fopenmp", "-I", CSRC, "-I", os.path.join(REPO, "include"), str(src),
                    os.path.join(CSRC, "fe_data.cpp"), "-o", str(exe)], check=True)
    return exe


@pytest.mark.parametrize("ck", [16, 32])
def test_patch_gemm_image_reproduces_the_patch_solve(harness, ck):
    out = subprocess.run([str(harness), str(ck)], capture_output=True, text=True, check=True).stdout.split()
    rows = [out[i:i + 3] for i in range(0, len(out), 3)]
    assert [int(r[0]) for r in rows] == [2, 3, 4]
    for k, err, pad in rows:
        # the image is rounded to TF32 (10 mantissa bits): ~1e-4 of the largest entry
        assert float(err) < 1e-3, (k, err)
        assert float(pad) == 0.0, (k, pad)
