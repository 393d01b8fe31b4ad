// Drives the C++ drop-in API (include/cytnx.hpp) the way example/DMRG/dmrg_two_sites_U1.py
// drives the reference's: bonds with U(1) charges, BlockUniTensors, the two-site H_eff as a
// Network inside a LinOp subclass, linalg::Lanczos(method "Gnd"); plus Tensor
// permute/contiguous and linalg::Tensordot.  Inputs come from a binary file written by
// tests/test_cxx_api.py; the results go to a binary file that the test compares with the
// oracle.
//
//   two_site_lanczos <in.bin> <out.bin>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

#include "cytnx.hpp"

using namespace cytnx;

namespace {
struct Reader {
  std::ifstream f;
  explicit Reader(const char *p) : f(p, std::ios::binary) {
    if (!f) throw std::runtime_error("cannot open input");
  }
  int64_t i64() {
    int64_t v;
    f.read((char *)&v, 8);
    return v;
  }
  std::vector<int64_t> i64s(int64_t n) {
    std::vector<int64_t> v(n);
    f.read((char *)v.data(), 8 * n);
    return v;
  }
  std::vector<double> f64s(int64_t n) {
    std::vector<double> v(n);
    f.read((char *)v.data(), 8 * n);
    return v;
  }
};

// the effective Hamiltonian of example/DMRG/dmrg_two_sites_U1.py:10-23
class Hxx : public LinOp {
 public:
  Network anet;
  Hxx(cytnx_uint64 psidim, const UniTensor &L, const UniTensor &M1, const UniTensor &M2, const UniTensor &R)
      : LinOp("mv", psidim, Type.Double, Device.cuda) {
    anet.FromString({"psi: -1,-2,-3,-4", "L: -5,-1,0", "R: -7,-4,3", "M1: -5,-6,-2,1", "M2: -6,-7,-3,2",
                     "TOUT: 0,1;2,3"});
    anet.PutUniTensors({"L", "M1", "M2", "R"}, {L, M1, M2, R});
  }
  UniTensor matvec(const UniTensor &v) override {
    anet.PutUniTensor("psi", v);
    UniTensor out = anet.Launch();
    out.relabel_(v.labels());
    return out;
  }
  using LinOp::matvec;
};
}  // namespace

int main(int argc, char **argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
    return 2;
  }
  try {
    Reader in(argv[1]);
    const int64_t nsec = in.i64();
    const auto q = in.i64s(nsec), d = in.i64s(nsec);
    std::vector<std::vector<cytnx_int64>> qn;
    std::vector<cytnx_uint64> dg;
    for (int64_t i = 0; i < nsec; ++i) {
      qn.push_back({q[i]});
      dg.push_back((cytnx_uint64)d[i]);
    }
    const Bond V(BD_KET, qn, dg, {Symmetry::U1()});
    const Bond phys(BD_KET, {{1}, {-1}}, {1, 1});
    const Bond inner(BD_KET, {{0}, {-2}, {2}, {0}, {0}}, {1, 1, 1, 1, 1});
    UniTensor M({inner, inner.redirect(), phys, phys.redirect()}, {"w0", "w1", "s", "sp"}, 2);
    const int64_t nmpo = in.i64();
    for (int64_t t = 0; t < nmpo; ++t) {
      const auto idx = in.i64s(4);
      const auto val = in.f64s(1);
      M.put_block(Tensor::from_vector(val, {1, 1, 1, 1}), std::vector<cytnx_int64>(idx.begin(), idx.end()));
    }
    UniTensor L({inner.redirect(), V.redirect(), V}, {"w", "a", "ap"}, 1);
    UniTensor R({inner, V, V.redirect()}, {"w", "b", "bp"}, 1);
    UniTensor psi({V, phys.redirect(), phys.redirect(), V.redirect()}, {"a", "s1", "s2", "b"}, 1);
    L.from_vector(in.f64s(in.i64()));
    R.from_vector(in.f64s(in.i64()));
    psi.from_vector(in.f64s(in.i64()));
    const int64_t maxiter = in.i64();

    Hxx H(psi.storage_size(), L, M, M, R);
    const UniTensor hpsi = H.matvec(psi);
    auto res = linalg::Lanczos(&H, psi, "Gnd", 1e-300, (unsigned int)maxiter);
    const double E = res[0].get_block().item();
    const std::vector<double> vec = res[1].to_vector();

    // Tensor permute + contiguous (all orders of a rank-4 tensor's first perm set) and Tensordot
    std::vector<double> a(4 * 3 * 5 * 2);
    for (size_t i = 0; i < a.size(); ++i) a[i] = (double)i;
    const Tensor T = Tensor::from_vector(a, {4, 3, 5, 2});
    const std::vector<double> perm = T.permute({3, 1, 0, 2}).contiguous().to_vector();
    const Tensor P2 = T.permute({2, 0, 3, 1}).permute({1, 0, 3, 2});  // lazy chain
    const std::vector<double> perm2 = P2.contiguous().to_vector();
    std::vector<double> b(5 * 2 * 6);
    for (size_t i = 0; i < b.size(); ++i) b[i] = 0.5 * (double)i - 7.0;
    const Tensor B = Tensor::from_vector(b, {5, 2, 6});
    const std::vector<double> td = linalg::Tensordot(T, B, {2, 3}, {0, 1}).to_vector();  // [4,3,6]

    // error path: BRA contracted with BRA throws cytnx::error
    int threw = 0;
    try {
      UniTensor X({V.redirect(), V}, {"x", "y"}, 1), Y({V.redirect(), V}, {"x", "z"}, 1);
      Contract(X, Y);
    } catch (const cytnx::error &) {
      threw = 1;
    }

    std::ofstream out(argv[2], std::ios::binary);
    auto w64 = [&](int64_t v) { out.write((const char *)&v, 8); };
    auto wvec = [&](const std::vector<double> &v) {
      w64((int64_t)v.size());
      out.write((const char *)v.data(), 8 * v.size());
    };
    wvec(hpsi.to_vector());
    out.write((const char *)&E, 8);
    wvec(vec);
    wvec(perm);
    wvec(perm2);
    wvec(td);
    w64(threw);
    std::printf("E = %.15f\n", E);
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
