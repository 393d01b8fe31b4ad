// C++ drop-in API (namespace cytnx, include/cytnx.hpp) over the C ABI of cytnx_b200.h.
//
// Host-side bookkeeping only: bonds, labels, block layouts, lazy permutations, contraction
// plans and device allocations.  Every computation is a ctn_* call (hand-written sm_100a
// kernels); the C ABI status is turned into cytnx::error with ctn_last_error()'s text.
// Device memory: stream-ordered allocations (cudaMallocAsync / cudaFreeAsync) on the legacy
// default stream, on which all work is issued.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <fstream>
#include <functional>
#include <mutex>
#include <numeric>
#include <set>
#include <sstream>
#include <unordered_map>

#include "../../include/cytnx.hpp"

namespace cytnx {

namespace {
void check(ctn_status st, const char *where) {
  if (st != CTN_OK) throw error(std::string("[ERROR][") + where + "] " + ctn_last_error());
}
void check_cuda(cudaError_t e, const char *where) {
  if (e != cudaSuccess) throw error(std::string("[ERROR][") + where + "] CUDA: " + cudaGetErrorString(e));
}
std::string join_labels(const std::vector<std::string> &v) {
  std::string s;
  for (size_t i = 0; i < v.size(); ++i) s += (i ? "," : "") + v[i];
  return s;
}
}  // namespace

// ------------------------------------------------------------------ Type
std::string Type_class::getname(unsigned int dtype) {
  static const char *names[] = {"Void",  "Complex Double (Complex Float64)", "Complex Float (Complex Float32)",
                                "Double (Float64)", "Float (Float32)", "Int64", "Uint64", "Int32", "Uint32",
                                "Int16", "Uint16", "Bool"};
  return dtype < 12 ? names[dtype] : "Unknown";
}
size_t Type_class::typeSize(unsigned int dtype) { return ctn_dtype_size((int)dtype); }

// ------------------------------------------------------------------ device buffers
namespace detail {
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  bool owned = true;
  int device = 0;
  DevBuf(size_t nbytes, int dev, bool zero) : bytes(nbytes), device(dev) {
    if (nbytes) {
      check_cuda(cudaSetDevice(dev), "alloc");
      check_cuda(cudaMallocAsync(&p, nbytes, 0), "alloc");
      if (zero) check_cuda(cudaMemsetAsync(p, 0, nbytes, 0), "alloc");
    }
  }
  DevBuf(void *external, size_t nbytes, int dev) : p(external), bytes(nbytes), owned(false), device(dev) {}
  ~DevBuf() {
    if (owned && p) cudaFreeAsync(p, 0);
  }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
};

// Blocks of a block-sparse tensor with the given (stored-order) bonds: BlockUniTensor::Init
// enumeration (ctn_blocks_enumerate), back to back.
struct Layout {
  int rank = 0;
  int64_t nblocks = 0;
  std::vector<int64_t> itoi, shapes, offs, sizes;  // [nblocks][rank], [nblocks][rank], [nblocks], [nblocks]
  int64_t nelem = 0;
  std::map<std::vector<int64_t>, int64_t> index;
};
}  // namespace detail

namespace {
std::mutex g_mu;
std::map<std::string, std::shared_ptr<const detail::Layout>> g_layouts;  // kept for the process lifetime

std::shared_ptr<const detail::Layout> layout_for(const std::vector<Bond> &bonds) {
  std::string key;
  for (const auto &b : bonds) key += b.signature() + "|";
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_layouts.find(key);
    if (it != g_layouts.end()) return it->second;
  }
  auto L = std::make_shared<detail::Layout>();
  const int rank = (int)bonds.size();
  L->rank = rank;
  const int nsym = (int)bonds[0].Nsym();
  std::vector<int32_t> stype(nsym), btype(rank);
  std::vector<int64_t> symn(nsym), nqs(rank);
  for (int s = 0; s < nsym; ++s) {
    stype[s] = bonds[0].syms()[s].stype();
    symn[s] = bonds[0].syms()[s].n();
  }
  std::vector<std::vector<int64_t>> tabs(rank);
  std::vector<const int64_t *> ptrs(rank);
  int64_t cap = 1;
  for (int i = 0; i < rank; ++i) {
    btype[i] = bonds[i].type() == BD_BRA ? 1 : -1;
    nqs[i] = (int64_t)bonds[i].Nqnum();
    cap *= std::max<int64_t>(1, nqs[i]);
    for (const auto &q : bonds[i].qnums()) tabs[i].insert(tabs[i].end(), q.begin(), q.end());
    ptrs[i] = tabs[i].data();
  }
  std::vector<int64_t> itoi((size_t)cap * rank);
  int64_t count = 0;
  check(ctn_blocks_enumerate(rank, nsym, stype.data(), symn.data(), btype.data(), nqs.data(), ptrs.data(),
                             itoi.data(), cap, &count),
        "BlockUniTensor::Init");
  itoi.resize((size_t)count * rank);
  L->nblocks = count;
  L->itoi = itoi;
  L->shapes.resize(itoi.size());
  L->offs.resize(count);
  L->sizes.resize(count);
  int64_t off = 0;
  for (int64_t b = 0; b < count; ++b) {
    int64_t sz = 1;
    for (int i = 0; i < rank; ++i) {
      const int64_t d = (int64_t)bonds[i].getDegeneracies()[itoi[b * rank + i]];
      L->shapes[b * rank + i] = d;
      sz *= d;
    }
    L->offs[b] = off;
    L->sizes[b] = sz;
    off += sz;
    L->index[std::vector<int64_t>(itoi.begin() + b * rank, itoi.begin() + (b + 1) * rank)] = b;
  }
  L->nelem = off;
  std::lock_guard<std::mutex> lk(g_mu);
  auto ins = g_layouts.emplace(key, L);
  return ins.first->second;
}

// device scalar constants for the BLAS-1 entry points (per device, never freed)
const double *device_one(int dev) {
  static std::mutex mu;
  static std::map<int, double *> ones;
  std::lock_guard<std::mutex> lk(mu);
  auto it = ones.find(dev);
  if (it != ones.end()) return it->second;
  double *p = nullptr;
  check_cuda(cudaMalloc(&p, sizeof(double)), "constant");
  const double one = 1.0;
  check_cuda(cudaMemcpy(p, &one, sizeof(double), cudaMemcpyHostToDevice), "constant");
  ones[dev] = p;
  return p;
}

// ------------------------------------------------------------------ contraction plans
struct PlanHolder {
  ctn_contract_plan *h = nullptr;
  size_t scratch_bytes = 0;
  std::shared_ptr<detail::DevBuf> scratch;
  std::vector<std::vector<int64_t>> keep;
  ~PlanHolder() {
    if (h) ctn_contract_plan_destroy(h);
  }
};
std::map<std::string, std::shared_ptr<PlanHolder>> g_plans;

std::string vec_key(const std::vector<int64_t> &v) {
  std::string s;
  for (auto x : v) s += std::to_string(x) + ",";
  return s;
}

struct DescData {
  std::vector<int64_t> itoi, shapes, offs, perm;
  int rank = 0;
  int64_t nblocks = 0;
  ctn_block_desc desc() const {
    ctn_block_desc d;
    d.rank = rank;
    d.nblocks = nblocks;
    d.itoi = itoi.data();
    d.shapes = shapes.data();
    d.offs = offs.data();
    d.perm = perm.empty() ? nullptr : perm.data();
    return d;
  }
};

// descriptor of a stored layout seen through the lazy mapper (logical tuples and shapes)
DescData block_desc(const detail::Layout &L, const std::vector<cytnx_uint64> &mapper) {
  DescData d;
  d.rank = L.rank;
  d.nblocks = L.nblocks;
  d.itoi.resize(L.itoi.size());
  d.shapes.resize(L.shapes.size());
  for (int64_t b = 0; b < L.nblocks; ++b)
    for (int i = 0; i < L.rank; ++i) {
      d.itoi[b * L.rank + i] = L.itoi[b * L.rank + mapper[i]];
      d.shapes[b * L.rank + i] = L.shapes[b * L.rank + mapper[i]];
    }
  d.offs = L.offs;
  bool ident = true;
  for (int i = 0; i < L.rank; ++i) ident = ident && mapper[i] == (cytnx_uint64)i;
  if (!ident) d.perm.assign(mapper.begin(), mapper.end());
  return d;
}

DescData dense_desc(const std::vector<cytnx_uint64> &shape, const std::vector<cytnx_uint64> &mapper) {
  DescData d;
  d.rank = (int)shape.size();
  d.nblocks = 1;
  d.itoi.assign(d.rank, 0);
  d.shapes.assign(shape.begin(), shape.end());
  d.offs.assign(1, 0);
  bool ident = true;
  for (int i = 0; i < d.rank; ++i) ident = ident && mapper[i] == (cytnx_uint64)i;
  if (!ident) d.perm.assign(mapper.begin(), mapper.end());
  return d;
}

std::shared_ptr<PlanHolder> get_plan(const std::string &key, const DescData &A, const DescData &B,
                                     const std::vector<int64_t> &c1, const std::vector<int64_t> &c2,
                                     const DescData &O) {
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_plans.find(key);
    if (it != g_plans.end()) return it->second;
  }
  auto P = std::make_shared<PlanHolder>();
  const ctn_block_desc dA = A.desc(), dB = B.desc(), dO = O.desc();
  check(ctn_contract_plan_create(&dA, &dB, (int)c1.size(), c1.data(), c2.data(), &dO, &P->h),
        "BlockUniTensor::contract");
  P->scratch_bytes = ctn_contract_plan_scratch_bytes(P->h);
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_plans.size() >= 512) g_plans.clear();  // bounded: plans are rebuilt on demand
  g_plans[key] = P;
  return P;
}

void run_plan(PlanHolder &P, const void *a, const void *b, void *out, int dev) {
  if (!P.scratch || P.scratch->bytes < std::max<size_t>(P.scratch_bytes, 16))
    P.scratch = std::make_shared<detail::DevBuf>(std::max<size_t>(P.scratch_bytes, 16), dev, false);
  check(ctn_contract_execute(P.h, CTN_FLOAT64, a, b, out, P.scratch->p, nullptr), "contract");
}
}  // namespace

// ------------------------------------------------------------------ Bond
Bond::Bond(const cytnx_uint64 &dim, const bondType &bd_type) : dim_(dim), type_(bd_type) {}

Bond::Bond(const bondType &bd_type, const std::vector<std::vector<cytnx_int64>> &in_qnums,
           const std::vector<cytnx_uint64> &degs, const std::vector<Symmetry> &in_syms)
    : type_(bd_type), qnums_(in_qnums), degs_(degs), syms_(in_syms) {
  if (bd_type == BD_REG) throw error("[ERROR][Bond] a bond with quantum numbers must be BD_KET or BD_BRA.");
  if (in_qnums.size() != degs.size()) throw error("[ERROR][Bond] qnums and degs have different lengths.");
  const size_t nsym = in_qnums.empty() ? 0 : in_qnums[0].size();
  for (const auto &q : in_qnums)
    if (q.size() != nsym) throw error("[ERROR][Bond] every qnum needs one value per symmetry.");
  if (syms_.empty()) syms_.assign(nsym, Symmetry::U1());
  if (syms_.size() != nsym) throw error("[ERROR][Bond] number of symmetries does not match the qnums.");
  dim_ = 0;
  for (auto d : degs) dim_ += d;
}

Bond Bond::redirect() const {
  Bond b = *this;
  b.type_ = type_ == BD_KET ? BD_BRA : type_ == BD_BRA ? BD_KET : BD_REG;
  return b;
}
Bond &Bond::redirect_() {
  *this = redirect();
  return *this;
}
bool Bond::operator==(const Bond &o) const {
  return dim_ == o.dim_ && type_ == o.type_ && qnums_ == o.qnums_ && degs_ == o.degs_ && syms_ == o.syms_;
}
std::string Bond::signature() const {
  std::ostringstream s;
  s << (int)type_ << ":" << dim_ << ":";
  for (const auto &y : syms_) s << y.stype() << "/" << y.n() << ";";
  for (size_t i = 0; i < degs_.size(); ++i) {
    for (auto q : qnums_[i]) s << q << ",";
    s << "x" << degs_[i] << ";";
  }
  return s.str();
}

// ------------------------------------------------------------------ Tensor
static std::vector<cytnx_uint64> iota_u64(size_t n) {
  std::vector<cytnx_uint64> v(n);
  std::iota(v.begin(), v.end(), 0);
  return v;
}

Tensor::Tensor(const std::vector<cytnx_uint64> &shape, const unsigned int &dtype, const int &device,
               const bool &init_zero)
    : shape_(shape), mapper_(iota_u64(shape.size())), invmapper_(iota_u64(shape.size())), dtype_(dtype),
      device_(device) {
  if (device < 0) throw error("[ERROR][Tensor] storage lives on a CUDA device (Device.cuda + i).");
  if (Type.typeSize(dtype) == 0) throw error("[ERROR][Tensor] invalid dtype.");
  buf_ = std::make_shared<detail::DevBuf>(size() * Type.typeSize(dtype), device, init_zero);
}

Tensor Tensor::from_host(const void *data, const std::vector<cytnx_uint64> &shape, const unsigned int &dtype,
                         const int &device) {
  Tensor t(shape, dtype, device, false);
  if (t.size())
    check_cuda(cudaMemcpy(t.buf_->p, data, t.size() * Type.typeSize(dtype), cudaMemcpyHostToDevice), "Tensor");
  return t;
}
Tensor Tensor::from_vector(const std::vector<double> &v, const std::vector<cytnx_uint64> &shape,
                           const int &device) {
  Tensor t(shape, Type.Double, device, false);
  if (t.size() != v.size()) throw error("[ERROR][Tensor] vector size does not match the shape.");
  if (t.size()) check_cuda(cudaMemcpy(t.buf_->p, v.data(), v.size() * 8, cudaMemcpyHostToDevice), "Tensor");
  return t;
}

Tensor Tensor::from_device(void *ptr, const std::vector<cytnx_uint64> &shape, const unsigned int &dtype,
                           const int &device) {
  Tensor t;
  t.shape_ = shape;
  t.mapper_ = iota_u64(shape.size());
  t.invmapper_ = t.mapper_;
  t.dtype_ = dtype;
  t.device_ = device;
  t.buf_ = std::make_shared<detail::DevBuf>(ptr, t.size() * Type.typeSize(dtype), device);
  return t;
}

cytnx_uint64 Tensor::size() const {
  cytnx_uint64 n = 1;
  for (auto s : shape_) n *= s;
  return n;
}
bool Tensor::is_contiguous() const {
  for (size_t i = 0; i < mapper_.size(); ++i)
    if (mapper_[i] != i) return false;
  return true;
}
void *Tensor::device_ptr() const {
  if (!buf_) throw error("[ERROR][Tensor] empty tensor.");
  return (char *)buf_->p + offset_ * Type.typeSize(dtype_);
}

Tensor Tensor::permute(const std::vector<cytnx_uint64> &rnks) const {
  Tensor t = *this;
  t.permute_(rnks);
  return t;
}
Tensor &Tensor::permute_(const std::vector<cytnx_uint64> &rnks) {
  const size_t r = shape_.size();
  if (rnks.size() != r) throw error("[ERROR][Tensor::permute] the number of indices does not match the rank.");
  std::vector<bool> seen(r, false);
  for (auto x : rnks) {
    if (x >= r || seen[x]) throw error("[ERROR][Tensor::permute] invalid permutation.");
    seen[x] = true;
  }
  std::vector<cytnx_uint64> fwd(r), shp(r), inv(r);
  for (size_t i = 0; i < r; ++i) {
    fwd[i] = mapper_[rnks[i]];
    shp[i] = shape_[rnks[i]];
  }
  for (size_t i = 0; i < r; ++i) inv[fwd[i]] = i;
  mapper_ = fwd;
  invmapper_ = inv;
  shape_ = shp;
  return *this;
}

Tensor Tensor::contiguous() const {
  if (is_contiguous()) return *this;
  const size_t r = shape_.size();
  std::vector<uint64_t> oldshape(r);
  for (size_t i = 0; i < r; ++i) oldshape[i] = shape_[invmapper_[i]];
  Tensor out(shape_, dtype_, device_, false);
  if (size())
    check(ctn_permute(device_ptr(), out.buf_->p, (int)dtype_, (int)r, oldshape.data(), mapper_.data(), nullptr),
          "Tensor::contiguous");
  return out;
}
Tensor &Tensor::contiguous_() {
  *this = contiguous();
  return *this;
}
Tensor Tensor::reshape(const std::vector<cytnx_int64> &new_shape) const {
  Tensor t = contiguous();
  t.reshape_(new_shape);
  return t;
}
Tensor &Tensor::reshape_(const std::vector<cytnx_int64> &new_shape) {
  if (!is_contiguous()) contiguous_();
  cytnx_int64 known = 1, neg = -1;
  for (size_t i = 0; i < new_shape.size(); ++i) {
    if (new_shape[i] == -1) {
      if (neg >= 0) throw error("[ERROR][Tensor::reshape] only one -1 is allowed.");
      neg = (cytnx_int64)i;
    } else {
      known *= new_shape[i];
    }
  }
  std::vector<cytnx_uint64> s(new_shape.size());
  for (size_t i = 0; i < s.size(); ++i) s[i] = (cytnx_uint64)new_shape[i];
  if (neg >= 0) {
    if (known == 0 || size() % (cytnx_uint64)known) throw error("[ERROR][Tensor::reshape] size mismatch.");
    s[neg] = size() / (cytnx_uint64)known;
  }
  cytnx_uint64 n = 1;
  for (auto x : s) n *= x;
  if (n != size()) throw error("[ERROR][Tensor::reshape] size mismatch.");
  shape_ = s;
  mapper_ = iota_u64(s.size());
  invmapper_ = mapper_;
  return *this;
}
Tensor Tensor::clone() const {
  Tensor c = contiguous();
  if (c.buf_ != buf_ || c.offset_ != offset_) return c;
  Tensor out(shape_, dtype_, device_, false);
  if (size())
    check_cuda(cudaMemcpyAsync(out.buf_->p, device_ptr(), size() * Type.typeSize(dtype_), cudaMemcpyDeviceToDevice, 0),
               "Tensor::clone");
  return out;
}
void Tensor::to_host(void *dst) const {
  Tensor c = contiguous();
  if (size())
    check_cuda(cudaMemcpy(dst, c.device_ptr(), size() * Type.typeSize(dtype_), cudaMemcpyDeviceToHost), "Tensor");
}
std::vector<double> Tensor::to_vector() const {
  if (dtype_ != Type.Double) throw error("[ERROR][Tensor::to_vector] Double tensors only.");
  std::vector<double> v(size());
  to_host(v.data());
  return v;
}
double Tensor::item() const {
  if (size() != 1) throw error("[ERROR][Tensor::item] the tensor has more than one element.");
  return to_vector()[0];
}

// ------------------------------------------------------------------ UniTensor
static std::vector<std::string> default_labels(size_t r) {
  std::vector<std::string> l(r);
  for (size_t i = 0; i < r; ++i) l[i] = std::to_string(i);
  return l;
}
static void check_labels(const std::vector<std::string> &labels, size_t r) {
  if (labels.size() != r) throw error("[ERROR] labels must have same length as # of bonds.");
  std::vector<std::string> s = labels;
  std::sort(s.begin(), s.end());
  if (std::adjacent_find(s.begin(), s.end()) != s.end()) throw error("[ERROR] labels cannot contain duplicated elements.");
}

UniTensor::UniTensor(const std::vector<Bond> &bonds, const std::vector<std::string> &in_labels,
                     const cytnx_int64 &rowrank, const unsigned int &dtype, const int &device, const bool &is_diag,
                     const std::string &name)
    : bonds_(bonds), is_diag_(is_diag), name_(name), device_(device) {
  const size_t r = bonds.size();
  labels_ = in_labels.empty() ? default_labels(r) : in_labels;
  check_labels(labels_, r);
  if (dtype != Type.Double) throw error("[ERROR][UniTensor] the device contraction engine computes in Double.");
  bool sym = r > 0, any = false;
  for (const auto &b : bonds) {
    sym = sym && b.has_qnums();
    any = any || b.has_qnums();
  }
  if (sym) {
    block_ = true;
    for (const auto &b : bonds)
      if (b.syms() != bonds[0].syms()) throw error("[ERROR][BlockUniTensor] symmetry mismatch between bonds.");
    cytnx_int64 nket = 0;
    for (const auto &b : bonds) nket += b.type() == BD_KET;
    rowrank_ = rowrank < 0 ? nket : rowrank;
    if (rowrank_ > (cytnx_int64)r) throw error("[ERROR][BlockUniTensor] rowrank must be >=0 and <=rank.");
    layout_ = layout_for(bonds_);
    mapper_ = iota_u64(r);
    buf_ = std::make_shared<detail::DevBuf>((size_t)layout_->nelem * 8, device, true);
  } else {
    if (any) throw error("[ERROR] cannot mix symmetric and regular bonds.");
    std::vector<cytnx_uint64> shape;
    for (const auto &b : bonds) shape.push_back(b.dim());
    if (is_diag) shape = {bonds.empty() ? 0 : bonds[0].dim()};
    dense_ = Tensor(shape, dtype, device, true);
    rowrank_ = rowrank < 0 ? (is_diag ? 1 : (cytnx_int64)r / 2) : rowrank;
  }
}

UniTensor::UniTensor(const Tensor &in_tensor, const bool &is_diag, const cytnx_int64 &rowrank,
                     const std::vector<std::string> &in_labels, const std::string &name)
    : is_diag_(is_diag), name_(name), device_(in_tensor.device()), dense_(in_tensor) {
  for (auto s : in_tensor.shape()) bonds_.push_back(Bond(s));
  if (is_diag) bonds_ = {Bond(in_tensor.shape()[0]), Bond(in_tensor.shape()[0])};
  labels_ = in_labels.empty() ? default_labels(bonds_.size()) : in_labels;
  check_labels(labels_, bonds_.size());
  rowrank_ = rowrank < 0 ? (is_diag ? 1 : (cytnx_int64)bonds_.size() / 2) : rowrank;
}

std::vector<cytnx_uint64> UniTensor::shape() const {
  std::vector<cytnx_uint64> s;
  for (const auto &b : bonds_) s.push_back(b.dim());
  return s;
}
cytnx_uint64 UniTensor::Nblocks() const { return block_ ? (cytnx_uint64)layout_->nblocks : 1; }
bool UniTensor::is_contiguous() const {
  if (!block_) return dense_.is_contiguous();
  for (size_t i = 0; i < mapper_.size(); ++i)
    if (mapper_[i] != i) return false;
  return true;
}
std::vector<std::vector<cytnx_uint64>> UniTensor::get_itoi() const {
  std::vector<std::vector<cytnx_uint64>> out;
  if (!block_) return {std::vector<cytnx_uint64>(rank(), 0)};
  for (int64_t b = 0; b < layout_->nblocks; ++b) {
    std::vector<cytnx_uint64> t(rank());
    for (size_t i = 0; i < rank(); ++i) t[i] = (cytnx_uint64)layout_->itoi[b * layout_->rank + mapper_[i]];
    out.push_back(t);
  }
  return out;
}
std::vector<Bond> UniTensor::stored_bonds() const {
  std::vector<Bond> s(bonds_.size());
  for (size_t i = 0; i < bonds_.size(); ++i) s[mapper_[i]] = bonds_[i];
  return s;
}

UniTensor &UniTensor::set_rowrank_(const cytnx_uint64 &new_rowrank) {
  if (new_rowrank > rank()) throw error("[ERROR][UniTensor] rowrank cannot exceed the rank.");
  rowrank_ = (cytnx_int64)new_rowrank;
  return *this;
}
UniTensor UniTensor::set_rowrank(const cytnx_uint64 &new_rowrank) const {
  UniTensor u = *this;
  u.set_rowrank_(new_rowrank);
  return u;
}
UniTensor &UniTensor::set_labels(const std::vector<std::string> &new_labels) { return relabel_(new_labels); }
UniTensor &UniTensor::relabel_(const std::vector<std::string> &new_labels) {
  check_labels(new_labels, rank());
  labels_ = new_labels;
  return *this;
}
UniTensor UniTensor::relabel(const std::vector<std::string> &new_labels) const {
  UniTensor u = *this;
  u.relabel_(new_labels);
  return u;
}
UniTensor &UniTensor::relabel_(const std::string &old_label, const std::string &new_label) {
  auto it = std::find(labels_.begin(), labels_.end(), old_label);
  if (it == labels_.end()) throw error("[ERROR][UniTensor::relabel] label '" + old_label + "' not found.");
  std::vector<std::string> l = labels_;
  l[it - labels_.begin()] = new_label;
  return relabel_(l);
}
UniTensor UniTensor::relabel(const std::string &old_label, const std::string &new_label) const {
  UniTensor u = *this;
  u.relabel_(old_label, new_label);
  return u;
}

UniTensor UniTensor::permute(const std::vector<cytnx_int64> &mapper, const cytnx_int64 &rowrank) const {
  UniTensor u = *this;
  u.permute_(mapper, rowrank);
  return u;
}
UniTensor UniTensor::permute(const std::vector<std::string> &mapper, const cytnx_int64 &rowrank) const {
  UniTensor u = *this;
  u.permute_(mapper, rowrank);
  return u;
}
UniTensor &UniTensor::permute_(const std::vector<std::string> &mapper, const cytnx_int64 &rowrank) {
  std::vector<cytnx_int64> m;
  for (const auto &l : mapper) {
    auto it = std::find(labels_.begin(), labels_.end(), l);
    if (it == labels_.end()) throw error("[ERROR][UniTensor::permute] label '" + l + "' not found.");
    m.push_back(it - labels_.begin());
  }
  return permute_(m, rowrank);
}
UniTensor &UniTensor::permute_(const std::vector<cytnx_int64> &mapper, const cytnx_int64 &rowrank) {
  const size_t r = rank();
  if (mapper.size() != r) throw error("[ERROR][UniTensor::permute] the number of indices does not match the rank.");
  std::vector<bool> seen(r, false);
  for (auto x : mapper) {
    if (x < 0 || (size_t)x >= r || seen[x]) throw error("[ERROR][UniTensor::permute] invalid permutation.");
    seen[x] = true;
  }
  if (rowrank > (cytnx_int64)r) throw error("[ERROR][BlockUniTensor] rowrank cannot exceed the rank of UniTensor.");
  std::vector<Bond> nb(r);
  std::vector<std::string> nl(r);
  for (size_t i = 0; i < r; ++i) {
    nb[i] = bonds_[mapper[i]];
    nl[i] = labels_[mapper[i]];
  }
  if (block_) {
    std::vector<cytnx_uint64> nm(r);
    for (size_t i = 0; i < r; ++i) nm[i] = mapper_[mapper[i]];
    mapper_ = nm;
  } else if (!is_diag_) {
    std::vector<cytnx_uint64> m(mapper.begin(), mapper.end());
    dense_.permute_(m);
  }
  bonds_ = nb;
  labels_ = nl;
  if (rowrank >= 0) rowrank_ = rowrank;
  return *this;
}

UniTensor UniTensor::contiguous() const {
  if (is_contiguous()) return *this;
  UniTensor u = *this;
  if (!block_) {
    u.dense_ = dense_.contiguous();
    return u;
  }
  // blocks of the logical bonds in their own Init order; every stored block is permuted
  // into its place there (ctn_permute_blocks, one launch sequence)
  auto Ln = layout_for(bonds_);
  const int r = (int)rank();
  std::vector<int64_t> dst(layout_->nblocks);
  for (int64_t b = 0; b < layout_->nblocks; ++b) {
    std::vector<int64_t> t(r);
    for (int i = 0; i < r; ++i) t[i] = layout_->itoi[b * r + mapper_[i]];
    dst[b] = Ln->offs[Ln->index.at(t)];
  }
  std::vector<uint64_t> oldshapes(layout_->shapes.begin(), layout_->shapes.end());
  auto nbuf = std::make_shared<detail::DevBuf>((size_t)Ln->nelem * 8, device_, false);
  if (layout_->nblocks)
    check(ctn_permute_blocks(buf_->p, nbuf->p, CTN_FLOAT64, r, layout_->nblocks, oldshapes.data(),
                             layout_->offs.data(), dst.data(), mapper_.data(), nullptr),
          "BlockUniTensor::contiguous");
  u.layout_ = Ln;
  u.mapper_ = iota_u64(r);
  u.buf_ = nbuf;
  return u;
}
void UniTensor::contiguous_() { *this = contiguous(); }

Tensor UniTensor::get_block(const cytnx_uint64 &idx) const {
  if (!block_) return dense_.clone();
  if (idx >= Nblocks()) throw error("[ERROR][UniTensor::get_block] block index out of range.");
  const int r = (int)rank();
  std::vector<cytnx_uint64> stored_shape(r), logical(r);
  for (int i = 0; i < r; ++i) stored_shape[i] = (cytnx_uint64)layout_->shapes[idx * r + i];
  for (int i = 0; i < r; ++i) logical[i] = stored_shape[mapper_[i]];
  Tensor t;
  t.buf_ = buf_;
  t.offset_ = (cytnx_uint64)layout_->offs[idx];
  t.shape_ = stored_shape;
  t.mapper_ = iota_u64(r);
  t.invmapper_ = t.mapper_;
  t.dtype_ = Type.Double;
  t.device_ = device_;
  return t.permute(mapper_).clone();
}
Tensor UniTensor::get_block(const std::vector<cytnx_int64> &qidx) const {
  if (!block_) throw error("[ERROR][UniTensor::get_block] qnum indices need a block form tensor.");
  const int r = (int)rank();
  if ((int)qidx.size() != r) throw error("[ERROR][UniTensor::get_block] one qnum index per bond.");
  std::vector<int64_t> stored(r);
  for (int i = 0; i < r; ++i) stored[mapper_[i]] = qidx[i];
  auto it = layout_->index.find(stored);
  if (it == layout_->index.end()) throw error("[ERROR][UniTensor::get_block] no block with these qnum indices.");
  return get_block((cytnx_uint64)it->second);
}
void UniTensor::put_block(const Tensor &in, const cytnx_uint64 &idx) {
  if (!block_) {
    if (in.shape() != dense_.shape()) throw error("[ERROR][UniTensor::put_block] shape mismatch.");
    dense_ = in.clone();
    return;
  }
  contiguous_();
  if (idx >= Nblocks()) throw error("[ERROR][UniTensor::put_block] block index out of range.");
  const int r = (int)rank();
  std::vector<cytnx_uint64> shp(r);
  for (int i = 0; i < r; ++i) shp[i] = (cytnx_uint64)layout_->shapes[idx * r + i];
  if (in.shape() != shp) throw error("[ERROR][UniTensor::put_block] the block's shape does not match.");
  if (in.dtype() != Type.Double) throw error("[ERROR][UniTensor::put_block] Double blocks only.");
  Tensor c = in.contiguous();
  check_cuda(cudaMemcpyAsync((double *)buf_->p + layout_->offs[idx], c.device_ptr(), layout_->sizes[idx] * 8,
                             cudaMemcpyDeviceToDevice, 0),
             "UniTensor::put_block");
}
void UniTensor::put_block(const Tensor &in, const std::vector<cytnx_int64> &qidx) {
  contiguous_();
  std::vector<int64_t> t(qidx.begin(), qidx.end());
  auto it = layout_->index.find(t);
  if (it == layout_->index.end()) throw error("[ERROR][UniTensor::put_block] no block with these qnum indices.");
  put_block(in, (cytnx_uint64)it->second);
}

cytnx_uint64 UniTensor::storage_size() const { return block_ ? (cytnx_uint64)layout_->nelem : dense_.size(); }
double *UniTensor::storage_ptr() const {
  return block_ ? (double *)buf_->p : (double *)dense_.device_ptr();
}
std::vector<double> UniTensor::to_vector() const {
  UniTensor c = contiguous();
  std::vector<double> v(c.storage_size());
  if (!v.empty()) check_cuda(cudaMemcpy(v.data(), c.storage_ptr(), v.size() * 8, cudaMemcpyDeviceToHost), "UniTensor");
  return v;
}
void UniTensor::from_vector(const std::vector<double> &flat) {
  contiguous_();
  if (flat.size() != storage_size()) throw error("[ERROR][UniTensor::from_vector] size mismatch.");
  if (!flat.empty())
    check_cuda(cudaMemcpy(storage_ptr(), flat.data(), flat.size() * 8, cudaMemcpyHostToDevice), "UniTensor");
}
UniTensor UniTensor::view_of(double *device_flat) const {
  UniTensor u = *this;
  if (block_) {
    u.buf_ = std::make_shared<detail::DevBuf>(device_flat, (size_t)layout_->nelem * 8, device_);
  } else {
    Tensor t = dense_.contiguous();
    t.buf_ = std::make_shared<detail::DevBuf>(device_flat, t.size() * 8, device_);
    t.offset_ = 0;
    u.dense_ = t;
    if (!dense_.is_contiguous()) throw error("[ERROR][UniTensor::view_of] the template must be contiguous.");
  }
  return u;
}
UniTensor UniTensor::clone() const {
  UniTensor u = contiguous();
  if (!block_) {
    u.dense_ = u.dense_.clone();
    return u;
  }
  auto nbuf = std::make_shared<detail::DevBuf>((size_t)u.layout_->nelem * 8, device_, false);
  if (u.layout_->nelem)
    check_cuda(cudaMemcpyAsync(nbuf->p, u.buf_->p, u.layout_->nelem * 8, cudaMemcpyDeviceToDevice, 0), "clone");
  u.buf_ = nbuf;
  return u;
}
UniTensor UniTensor::Transpose() const {
  UniTensor u = *this;
  if (block_)
    for (auto &b : u.bonds_) b.redirect_();  // redirected bonds enumerate the same blocks
  std::vector<cytnx_int64> rev(rank());
  for (size_t i = 0; i < rank(); ++i) rev[i] = (cytnx_int64)(rank() - 1 - i);
  return u.permute(rev, (cytnx_int64)rank() - rowrank_);
}

Tensor UniTensor::Norm() const {
  Tensor out({1}, Type.Double, device_, false);
  const UniTensor c = contiguous();
  check(ctn_nrm2_f64(c.storage_ptr(), (int64_t)c.storage_size(), (double *)out.device_ptr(), nullptr), "Norm");
  return out;
}

void UniTensor::check_same_structure(const UniTensor &o, const char *where) const {
  if (block_ != o.block_ || rank() != o.rank()) throw error(std::string("[ERROR][") + where + "] structure mismatch.");
  for (size_t i = 0; i < rank(); ++i)
    if (bonds_[i].dim() != o.bonds_[i].dim() || bonds_[i].getDegeneracies() != o.bonds_[i].getDegeneracies())
      throw error(std::string("[ERROR][") + where + "] bond mismatch.");
}
UniTensor &UniTensor::operator+=(const UniTensor &rhs) {
  check_same_structure(rhs, "UniTensor::Add");
  *this = clone();
  const UniTensor r = rhs.contiguous();
  check(ctn_axpy_f64(r.storage_ptr(), storage_ptr(), (int64_t)storage_size(), device_one(device_), 1.0, nullptr),
        "UniTensor::Add");
  return *this;
}
UniTensor &UniTensor::operator-=(const UniTensor &rhs) {
  check_same_structure(rhs, "UniTensor::Sub");
  *this = clone();
  const UniTensor r = rhs.contiguous();
  check(ctn_axpy_f64(r.storage_ptr(), storage_ptr(), (int64_t)storage_size(), device_one(device_), -1.0, nullptr),
        "UniTensor::Sub");
  return *this;
}
UniTensor &UniTensor::operator*=(const double &a) {
  *this = clone();
  Tensor s = Tensor::from_vector({a}, {1}, device_);
  check(ctn_scal_f64(storage_ptr(), (int64_t)storage_size(), (const double *)s.device_ptr(), 0, nullptr),
        "UniTensor::Mul");
  return *this;
}
UniTensor &UniTensor::operator/=(const double &a) {
  *this = clone();
  Tensor s = Tensor::from_vector({a}, {1}, device_);
  check(ctn_scal_f64(storage_ptr(), (int64_t)storage_size(), (const double *)s.device_ptr(), 1, nullptr),
        "UniTensor::Div");
  return *this;
}
UniTensor UniTensor::operator+(const UniTensor &rhs) const {
  UniTensor u = *this;
  return u += rhs;
}
UniTensor UniTensor::operator-(const UniTensor &rhs) const {
  UniTensor u = *this;
  return u -= rhs;
}
UniTensor UniTensor::operator*(const double &a) const {
  UniTensor u = *this;
  return u *= a;
}
UniTensor UniTensor::operator/(const double &a) const {
  UniTensor u = *this;
  return u /= a;
}

UniTensor UniTensor::contract(const UniTensor &rhs, const bool &, const bool &) const { return Contract(*this, rhs); }

// ------------------------------------------------------------------ Contract
UniTensor Contract(const UniTensor &A, const UniTensor &B, const bool &, const bool &) {
  if (A.block_ != B.block_)
    throw error("[ERROR][contract] Cannot contract BlockUniTensor with other type of UniTensor.");
  // vec_intersect_: common labels in sorted order
  std::vector<std::string> la = A.labels_, lb = B.labels_;
  std::sort(la.begin(), la.end());
  std::sort(lb.begin(), lb.end());
  std::vector<std::string> comm;
  std::set_intersection(la.begin(), la.end(), lb.begin(), lb.end(), std::back_inserter(comm));
  std::vector<int64_t> c1, c2, n1, n2;
  for (const auto &l : comm) {
    c1.push_back(std::find(A.labels_.begin(), A.labels_.end(), l) - A.labels_.begin());
    c2.push_back(std::find(B.labels_.begin(), B.labels_.end(), l) - B.labels_.begin());
  }
  for (int64_t i = 0; i < (int64_t)A.rank(); ++i)
    if (std::find(c1.begin(), c1.end(), i) == c1.end()) n1.push_back(i);
  for (int64_t i = 0; i < (int64_t)B.rank(); ++i)
    if (std::find(c2.begin(), c2.end(), i) == c2.end()) n2.push_back(i);
  for (size_t k = 0; k < comm.size(); ++k) {
    const Bond &ba = A.bonds_[c1[k]], &bb = B.bonds_[c2[k]];
    if (A.block_) {
      if (ba.syms() != bb.syms())
        throw error("[ERROR][BlockUniTensor][contract] Two UniTensor have different symmetry types, cannot contract.");
      if ((int)ba.type() + (int)bb.type() != 0)
        throw error("[ERROR][BlockUniTensor][contract] A bond with type BRA can only be contracted with type KET. "
                    "Invalid contraction for label '" + comm[k] + "'.");
      if (ba.qnums() != bb.qnums() || ba.getDegeneracies() != bb.getDegeneracies())
        throw error("[ERROR][BlockUniTensor][contract] Contracted bond with label '" + comm[k] +
                    "' has a qnum/degeneracy mismatch.");
    } else if (ba.dim() != bb.dim()) {
      throw error("[ERROR][contract] dimension mismatch on label '" + comm[k] + "'");
    }
  }
  if (comm.empty()) throw error("[ERROR][contract] no common label: outer products are not supported here.");
  const int dev = A.device_;
  if (n1.empty() && n2.empty()) {  // every leg contracted: sum of block dot products
    std::vector<std::string> order;
    for (auto i : c1) order.push_back(A.labels_[i]);
    const UniTensor Ap = A.permute(std::vector<cytnx_int64>(c1.begin(), c1.end())).contiguous();
    const UniTensor Bp = B.permute(order).contiguous();
    Tensor out({1}, Type.Double, dev, true);
    if (!A.block_ || Ap.layout_->itoi == Bp.layout_->itoi) {
      check(ctn_dot_f64(Ap.storage_ptr(), Bp.storage_ptr(), (int64_t)Ap.storage_size(), (double *)out.device_ptr(),
                        nullptr),
            "contract");
    } else {
      double s = 0.0;
      for (int64_t a = 0; a < Ap.layout_->nblocks; ++a) {
        std::vector<int64_t> t(Ap.layout_->itoi.begin() + a * Ap.layout_->rank,
                               Ap.layout_->itoi.begin() + (a + 1) * Ap.layout_->rank);
        auto it = Bp.layout_->index.find(t);
        if (it == Bp.layout_->index.end()) continue;
        check(ctn_dot_f64(Ap.storage_ptr() + Ap.layout_->offs[a], Bp.storage_ptr() + Bp.layout_->offs[it->second],
                          Ap.layout_->sizes[a], (double *)out.device_ptr(), nullptr),
              "contract");
        s += out.item();
      }
      out = Tensor::from_vector({s}, {1}, dev);
    }
    out.reshape_({1});
    return UniTensor(out, false, 0, {"0"});
  }
  std::vector<Bond> ob;
  std::vector<std::string> ol;
  for (auto i : n1) {
    ob.push_back(A.bonds_[i]);
    ol.push_back(A.labels_[i]);
  }
  for (auto i : n2) {
    ob.push_back(B.bonds_[i]);
    ol.push_back(B.labels_[i]);
  }
  cytnx_int64 rr = A.rowrank_ + B.rowrank_;
  for (auto i : c1) rr -= i < A.rowrank_;
  for (auto i : c2) rr -= i < B.rowrank_;
  UniTensor out;
  out.block_ = A.block_;
  out.bonds_ = ob;
  out.labels_ = ol;
  out.rowrank_ = rr;
  out.device_ = dev;
  if (A.block_) {
    auto Lo = layout_for(ob);
    std::vector<int64_t> ma(A.mapper_.begin(), A.mapper_.end()), mb(B.mapper_.begin(), B.mapper_.end());
    std::ostringstream key;
    key << "B" << (const void *)A.layout_.get() << "|" << vec_key(ma) << "|" << (const void *)B.layout_.get() << "|"
        << vec_key(mb) << "|" << vec_key(c1) << "|" << vec_key(c2) << "|" << (const void *)Lo.get();
    auto P = get_plan(key.str(), block_desc(*A.layout_, A.mapper_), block_desc(*B.layout_, B.mapper_), c1, c2,
                      block_desc(*Lo, iota_u64(ob.size())));
    out.layout_ = Lo;
    out.mapper_ = iota_u64(ob.size());
    out.buf_ = std::make_shared<detail::DevBuf>((size_t)Lo->nelem * 8, dev, false);
    run_plan(*P, A.buf_->p, B.buf_->p, out.buf_->p, dev);
    return out;
  }
  const auto sa = A.dense_.shape(), sb = B.dense_.shape();
  std::vector<cytnx_uint64> os;
  for (auto i : n1) os.push_back(sa[i]);
  for (auto i : n2) os.push_back(sb[i]);
  std::vector<int64_t> ma(A.dense_.mapper().begin(), A.dense_.mapper().end()),
      mb(B.dense_.mapper().begin(), B.dense_.mapper().end());
  std::vector<int64_t> ia(sa.begin(), sa.end()), ib(sb.begin(), sb.end());
  std::ostringstream key;
  key << "D" << vec_key(ia) << "|" << vec_key(ma) << "|" << vec_key(ib) << "|" << vec_key(mb) << "|" << vec_key(c1)
      << "|" << vec_key(c2);
  auto P = get_plan(key.str(), dense_desc(sa, A.dense_.mapper()), dense_desc(sb, B.dense_.mapper()), c1, c2,
                    dense_desc(os, iota_u64(os.size())));
  out.dense_ = Tensor(os, Type.Double, dev, false);
  // the dense storages in physical order (the plan applies the lazy mappers)
  run_plan(*P, A.dense_.device_ptr(), B.dense_.device_ptr(), out.dense_.device_ptr(), dev);
  return out;
}

// ------------------------------------------------------------------ LinOp
LinOp::LinOp(const std::string &type, const cytnx_uint64 &nx, const int &dtype, const int &device)
    : type_(type), nx_(nx), dtype_(dtype), device_(device) {
  if (type != "mv" && type != "mv_elem")
    throw error("[ERROR][LinOp] currently only type=\"mv\" (matvec) can be used.");
  if (dtype < 1 || dtype > 11) throw error("[ERROR] invalid dtype.");
}
Tensor LinOp::matvec(const Tensor &) { throw error("[ERROR][LinOp] matvec(Tensor) is not overridden."); }
UniTensor LinOp::matvec(const UniTensor &) { throw error("[ERROR][LinOp] matvec(UniTensor) is not overridden."); }

// ------------------------------------------------------------------ Network
static std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}
static std::vector<std::string> split_labels(const std::string &s) {
  std::vector<std::string> out;
  std::string cur;
  std::stringstream ss(s);
  while (std::getline(ss, cur, ',')) {
    cur = trim(cur);
    if (!cur.empty()) out.push_back(cur);
  }
  return out;
}

void Network::Fromfile(const std::string &fname) {
  std::ifstream f(fname);
  if (!f) throw error("[ERROR][Network] cannot open '" + fname + "'");
  std::vector<std::string> lines;
  std::string l;
  while (std::getline(f, l)) lines.push_back(l);
  FromString(lines);
}

void Network::FromString(const std::vector<std::string> &contents) {
  *this = Network();
  for (auto line : contents) {
    line = trim(line.substr(0, line.find('#')));
    if (line.empty()) continue;
    const size_t c = line.find(':');
    if (c == std::string::npos) throw error("[ERROR][Network] invalid line '" + line + "'");
    const std::string name = trim(line.substr(0, c)), rest = line.substr(c + 1);
    if (name == "TOUT") {
      const size_t sc = rest.find(';');
      std::vector<std::string> a = split_labels(rest.substr(0, sc)), b;
      if (sc != std::string::npos) b = split_labels(rest.substr(sc + 1));
      tout_ = a;
      tout_.insert(tout_.end(), b.begin(), b.end());
      tout_rowrank_ = (cytnx_int64)a.size();
    } else if (name == "ORDER") {
      order_ = trim(rest);
    } else {
      if (std::find(names_.begin(), names_.end(), name) != names_.end())
        throw error("[ERROR][Network] duplicated tensor name '" + name + "'");
      std::string r = rest;
      std::replace(r.begin(), r.end(), ';', ',');
      names_.push_back(name);
      labels_.push_back(split_labels(r));
    }
  }
  if (names_.empty()) throw error("[ERROR][Network] no tensor declared");
}

void Network::PutUniTensor(const std::string &name, const UniTensor &utensor,
                           const std::vector<std::string> &label_order) {
  auto it = std::find(names_.begin(), names_.end(), name);
  if (it == names_.end()) throw error("[ERROR][Network] no tensor named '" + name + "'");
  UniTensor u = label_order.empty() ? utensor : utensor.permute(label_order);
  const auto &labs = labels_[it - names_.begin()];
  if (u.rank() != labs.size())
    throw error("[ERROR][Network] tensor '" + name + "' rank does not match its " + std::to_string(labs.size()) +
                " labels");
  tensors_[name] = u.relabel(labs);
}
void Network::PutUniTensor(const cytnx_uint64 &idx, const UniTensor &utensor,
                           const std::vector<std::string> &label_order) {
  if (idx >= names_.size()) throw error("[ERROR][Network] tensor index out of range");
  PutUniTensor(names_[idx], utensor, label_order);
}
void Network::PutUniTensors(const std::vector<std::string> &names, const std::vector<UniTensor> &utensors) {
  if (names.size() != utensors.size()) throw error("[ERROR][Network] names and tensors differ in number");
  for (size_t i = 0; i < names.size(); ++i) PutUniTensor(names[i], utensors[i]);
}
void Network::RmUniTensor(const std::string &name) { tensors_.erase(name); }
void Network::setOrder(const bool &optimal, const std::string &contract_order) {
  optimal_ = optimal;
  if (!contract_order.empty()) order_ = contract_order;
}
std::string Network::getOrder() const {
  if (!order_.empty()) return order_;
  std::string s = names_[0];
  for (size_t i = 1; i < names_.size(); ++i) s = "(" + s + "," + names_[i] + ")";
  return s;
}

namespace {
// binary contraction tree: leaf = tensor index, node = (left, right)
struct Tree {
  int leaf = -1;
  std::shared_ptr<Tree> l, r;
};
std::shared_ptr<Tree> leaf(int i) {
  auto t = std::make_shared<Tree>();
  t->leaf = i;
  return t;
}
std::shared_ptr<Tree> node(std::shared_ptr<Tree> a, std::shared_ptr<Tree> b) {
  auto t = std::make_shared<Tree>();
  t->l = a;
  t->r = b;
  return t;
}
// ORDER grammar (src/contraction_tree.cpp:32-124): expr = name | "(" expr ("," expr)* ")", where a
// parenthesised list folds left
struct OrderParser {
  std::vector<std::string> toks;
  size_t pos = 0;
  const std::vector<std::string> &names;
  OrderParser(const std::string &s, const std::vector<std::string> &n) : names(n) {
    std::string cur;
    for (char ch : s) {
      if (ch == '(' || ch == ')' || ch == ',') {
        if (!trim(cur).empty()) toks.push_back(trim(cur));
        cur.clear();
        toks.push_back(std::string(1, ch));
      } else {
        cur += ch;
      }
    }
    if (!trim(cur).empty()) toks.push_back(trim(cur));
  }
  std::shared_ptr<Tree> expr() {
    if (pos >= toks.size()) throw error("[ERROR][Network] malformed ORDER");
    const std::string t = toks[pos++];
    if (t == "(") {
      auto acc = expr();
      while (pos < toks.size() && toks[pos] == ",") {
        ++pos;
        acc = node(acc, expr());
      }
      if (pos >= toks.size() || toks[pos] != ")") throw error("[ERROR][Network] malformed ORDER");
      ++pos;
      return acc;
    }
    auto it = std::find(names.begin(), names.end(), t);
    if (it == names.end()) throw error("[ERROR][Network] ORDER names unknown tensor '" + t + "'");
    return leaf((int)(it - names.begin()));
  }
};
}  // namespace

UniTensor Network::Launch() {
  for (const auto &n : names_)
    if (!tensors_.count(n)) throw error("[ERROR][Network] tensor '" + n + "' is not set");
  const int nt = (int)names_.size();
  std::shared_ptr<Tree> tree;
  if (nt == 1) {
    tree = leaf(0);
  } else if (!order_.empty()) {
    OrderParser p(order_, names_);
    tree = p.expr();
  } else if (optimal_) {
    // cheapest pairwise order on dense-equivalent cost (the role of SearchTree,
    // src/search_tree.cpp:9-150): dynamic programming over subsets
    std::map<std::string, double> dim;
    for (int i = 0; i < nt; ++i) {
      const UniTensor &u = tensors_.at(names_[i]);
      for (size_t k = 0; k < u.rank(); ++k) dim[u.labels_[k]] = (double)u.bonds_[k].dim();
    }
    const int full = (1 << nt) - 1;
    std::vector<double> cost(full + 1, 1e300);
    std::vector<std::set<std::string>> legs(full + 1);
    std::vector<std::shared_ptr<Tree>> best(full + 1);
    for (int i = 0; i < nt; ++i) {
      cost[1 << i] = 0.0;
      const UniTensor &u = tensors_.at(names_[i]);
      legs[1 << i] = std::set<std::string>(u.labels_.begin(), u.labels_.end());
      best[1 << i] = leaf(i);
    }
    for (int S = 1; S <= full; ++S) {
      if (__builtin_popcount(S) < 2) continue;
      for (int A = (S - 1) & S; A > 0; A = (A - 1) & S) {
        const int B = S ^ A;
        if (A > B || cost[A] >= 1e300 || cost[B] >= 1e300) continue;
        std::set<std::string> uni = legs[A];
        uni.insert(legs[B].begin(), legs[B].end());
        double c = 1.0;
        for (const auto &l : uni) c *= dim[l];
        const double tot = cost[A] + cost[B] + c;
        if (tot < cost[S]) {
          cost[S] = tot;
          best[S] = node(best[A], best[B]);
          std::set<std::string> out;
          for (const auto &l : uni)
            if (!(legs[A].count(l) && legs[B].count(l))) out.insert(l);
          legs[S] = out;
        }
      }
    }
    tree = best[full];
  } else {
    tree = leaf(0);
    for (int i = 1; i < nt; ++i) tree = node(tree, leaf(i));
  }
  std::function<UniTensor(const Tree &)> eval = [&](const Tree &t) -> UniTensor {
    if (t.leaf >= 0) return tensors_.at(names_[t.leaf]);
    return Contract(eval(*t.l), eval(*t.r));
  };
  UniTensor out = eval(*tree);
  if (!tout_.empty()) {
    std::vector<std::string> a = out.labels_, b = tout_;
    std::sort(a.begin(), a.end());
    std::sort(b.begin(), b.end());
    if (a != b) throw error("[ERROR][Network] TOUT labels do not match the result's labels");
    out = out.permute(tout_, tout_rowrank_);
  }
  return out;
}

// ------------------------------------------------------------------ linalg
namespace linalg {

Tensor Tensordot(const Tensor &Tl, const Tensor &Tr, const std::vector<cytnx_uint64> &idxl,
                 const std::vector<cytnx_uint64> &idxr, const bool &, const bool &) {
  if (idxl.size() != idxr.size()) throw error("[ERROR][Tensordot] idxl and idxr differ in length.");
  if (Tl.dtype() != Type.Double || Tr.dtype() != Type.Double)
    throw error("[ERROR][Tensordot] the device engine computes in Double.");
  std::vector<std::string> la(Tl.rank()), lb(Tr.rank());
  for (size_t i = 0; i < la.size(); ++i) la[i] = "l" + std::to_string(i);
  for (size_t i = 0; i < lb.size(); ++i) lb[i] = "r" + std::to_string(i);
  for (size_t k = 0; k < idxl.size(); ++k) {
    if (idxl[k] >= la.size() || idxr[k] >= lb.size()) throw error("[ERROR][Tensordot] index out of range.");
    // contracted pairs share a label; the label sorts in idxl order
    char buf[32];
    snprintf(buf, sizeof buf, "c%08zu", k);
    la[idxl[k]] = buf;
    lb[idxr[k]] = buf;
  }
  UniTensor A(Tl, false, 0, la), B(Tr, false, 0, lb);
  UniTensor C = Contract(A, B);
  return C.get_block();
}
Tensor Matmul(const Tensor &Tl, const Tensor &Tr) {
  if (Tl.rank() != 2 || Tr.rank() != 2) throw error("[ERROR][Matmul] rank-2 tensors only.");
  return Tensordot(Tl, Tr, {1}, {0});
}
Tensor Vectordot(const Tensor &Tl, const Tensor &Tr, const bool &) {
  if (Tl.size() != Tr.size()) throw error("[ERROR][Vectordot] size mismatch.");
  const Tensor a = Tl.contiguous(), b = Tr.contiguous();
  Tensor out({1}, Type.Double, Tl.device(), false);
  check(ctn_dot_f64((const double *)a.device_ptr(), (const double *)b.device_ptr(), (int64_t)a.size(),
                    (double *)out.device_ptr(), nullptr),
        "Vectordot");
  return out;
}
std::vector<Tensor> Tridiag(const Tensor &Diag, const Tensor &Sub_diag, const bool &is_V, const bool &is_row,
                            bool) {
  const std::vector<double> d = Diag.to_vector(), e = Sub_diag.to_vector();
  const int n = (int)d.size();
  if ((int)e.size() != std::max(n - 1, 0)) throw error("[ERROR][Tridiag] the sub-diagonal needs n - 1 elements.");
  std::vector<double> w(n), z(is_V ? (size_t)n * n : 0);
  check(ctn_tridiag_eigh(n, d.data(), e.data(), w.data(), is_V ? z.data() : nullptr), "Tridiag");
  std::vector<Tensor> out{Tensor::from_vector(w, {(cytnx_uint64)n}, Diag.device())};
  if (is_V) {
    Tensor Z = Tensor::from_vector(z, {(cytnx_uint64)n, (cytnx_uint64)n}, Diag.device());  // rows = eigenvectors
    out.push_back(is_row ? Z : Z.permute({1, 0}).contiguous());
  }
  return out;
}

namespace {
struct CbCtx {
  LinOp *op = nullptr;
  const UniTensor *ut = nullptr;
  const Tensor *t = nullptr;
  std::string err;
};
// matvec callback of the C-ABI Lanczos drivers: wrap x as the template's structure, call the
// user's LinOp, write its result (in the template's leg and block order) to y
int matvec_cb(void *user, const double *x, double *y, void *stream) {
  CbCtx *c = static_cast<CbCtx *>(user);
  try {
    if (c->ut) {
      UniTensor xin = c->ut->view_of(const_cast<double *>(x));
      UniTensor r = c->op->matvec(xin);
      if (r.labels() != c->ut->labels()) r = r.permute(c->ut->labels());
      r.contiguous_();
      if (r.storage_size() != c->ut->storage_size()) throw error("[ERROR][Lanczos] matvec changed the size.");
      if (r.get_itoi() != c->ut->get_itoi()) throw error("[ERROR][Lanczos] matvec changed the block structure.");
      check_cuda(cudaMemcpyAsync(y, r.storage_ptr(), r.storage_size() * 8, cudaMemcpyDeviceToDevice,
                                 (cudaStream_t)stream),
                 "Lanczos");
    } else {
      const Tensor xin = Tensor::from_device(const_cast<double *>(x), c->t->shape(), Type.Double, c->t->device());
      const Tensor r = c->op->matvec(xin).contiguous();
      if (r.size() != c->t->size() || r.dtype() != Type.Double)
        throw error("[ERROR][Lanczos] matvec must return a Double tensor of the input's size.");
      check_cuda(cudaMemcpyAsync(y, r.device_ptr(), r.size() * 8, cudaMemcpyDeviceToDevice, (cudaStream_t)stream),
                 "Lanczos");
    }
    return 0;
  } catch (const std::exception &e) {
    c->err = e.what();
    return 1;
  }
}
}  // namespace

std::vector<UniTensor> Lanczos(LinOp *Hop, const UniTensor &Tin, const std::string method, const double &CvgCrit,
                               const unsigned int &Maxiter, const cytnx_uint64 &k, const bool &is_V, const bool &,
                               const cytnx_uint32 &, const bool &) {
  if (method != "Gnd") throw error("[ERROR][Lanczos] method '" + method + "' is not supported (use \"Gnd\").");
  if (k != 1) throw error("[ERROR][Lanczos] the Gnd method returns the ground state only (k = 1).");
  if (!Hop) throw error("[ERROR][Lanczos] null LinOp.");
  if (Tin.rank() == 0) throw error("[ERROR][Lanczos] an initial UniTensor is required.");
  const UniTensor tmpl = Tin.contiguous();
  const int64_t n = (int64_t)tmpl.storage_size();
  if (Hop->nx() && (int64_t)Hop->nx() != n)
    throw error("[ERROR][Lanczos] the LinOp's nx does not match the initial vector.");
  const int dev = tmpl.device();
  const unsigned int maxiter = std::max(1u, Maxiter);
  detail::DevBuf kry((size_t)(maxiter + 1) * n * 8, dev, false), work((size_t)(4 * n + 64) * 8, dev, false);
  UniTensor vec = tmpl.clone();
  CbCtx ctx;
  ctx.op = Hop;
  ctx.ut = &tmpl;
  double E = 0.0;
  int iters = 0;
  const ctn_status st = ctn_lanczos_gnd(matvec_cb, &ctx, tmpl.storage_ptr(), n, (int)maxiter, CvgCrit,
                                        (double *)kry.p, (double *)work.p, vec.storage_ptr(), &E, &iters, nullptr);
  if (!ctx.err.empty()) throw error(ctx.err);
  check(st, "Lanczos");
  check_cuda(cudaStreamSynchronize(0), "Lanczos");
  std::vector<UniTensor> out{UniTensor(Tensor::from_vector({E}, {1}, dev), false, 0, {"0"})};
  if (is_V) out.push_back(vec);
  return out;
}

std::vector<Tensor> Lanczos(LinOp *Hop, const Tensor &Tin, const std::string method, const double &CvgCrit,
                            const unsigned int &Maxiter, const cytnx_uint64 &k, const bool &is_V, const bool &,
                            const cytnx_uint32 &, const bool &) {
  // Lanczos_Gnd (src/linalg/Lanczos_Gnd.cpp:16-134) on a flat Tensor
  if (method != "Gnd") throw error("[ERROR][Lanczos] method '" + method + "' is not supported (use \"Gnd\").");
  if (k != 1) throw error("[ERROR][Lanczos] the Gnd method returns the ground state only (k = 1).");
  if (!Hop) throw error("[ERROR][Lanczos] null LinOp.");
  if (Tin.dtype() != Type.Double) throw error("[ERROR][Lanczos] Double vectors only.");
  const Tensor tmpl = Tin.contiguous();
  const int64_t n = (int64_t)tmpl.size();
  if (Hop->nx() && (int64_t)Hop->nx() != n) throw error("[ERROR][Lanczos] the LinOp's nx does not match Tin.");
  const int dev = tmpl.device();
  const unsigned int maxiter = std::max(1u, Maxiter);
  detail::DevBuf kry((size_t)(maxiter + 1) * n * 8, dev, false), work((size_t)(4 * n + 64) * 8, dev, false);
  Tensor vec(tmpl.shape(), Type.Double, dev, false);
  CbCtx ctx;
  ctx.op = Hop;
  ctx.t = &tmpl;
  double E = 0.0;
  int iters = 0;
  const ctn_status st = ctn_lanczos_gnd(matvec_cb, &ctx, (const double *)tmpl.device_ptr(), n, (int)maxiter, CvgCrit,
                                        (double *)kry.p, (double *)work.p, (double *)vec.device_ptr(), &E, &iters,
                                        nullptr);
  if (!ctx.err.empty()) throw error(ctx.err);
  check(st, "Lanczos");
  check_cuda(cudaStreamSynchronize(0), "Lanczos");
  std::vector<Tensor> out{Tensor::from_vector({E}, {1}, dev)};
  if (is_V) out.push_back(vec);
  return out;
}

std::vector<UniTensor> Lanczos(LinOp *Hop, const UniTensor &Tin, const std::string which, const cytnx_uint64 &maxiter,
                               const cytnx_double &cvg_crit, const cytnx_uint64 &k, const bool &is_V,
                               const cytnx_int32 &ncv, const bool &) {
  int w;
  if (which == "SA")
    w = 0;
  else if (which == "LA")
    w = 1;
  else if (which == "LM")
    w = 2;
  else
    throw error("[ERROR][Lanczos] which must be \"SA\", \"LA\" or \"LM\".");
  if (!Hop) throw error("[ERROR][Lanczos] null LinOp.");
  const UniTensor tmpl = Tin.contiguous();
  const int64_t n = (int64_t)tmpl.storage_size();
  const int nc = ncv > 0 ? ncv : (int)std::min<int64_t>(n, 2 * (int64_t)k + 10);
  const int dev = tmpl.device();
  detail::DevBuf basis((size_t)(nc + 1) * n * 8, dev, false),
      work(ctn_lanczos_which_work_doubles(n, nc) * 8, dev, false), evecs(is_V ? (size_t)k * n * 8 : 8, dev, false);
  std::vector<double> evals(k);
  CbCtx ctx;
  ctx.op = Hop;
  ctx.ut = &tmpl;
  int iters = 0, nconv = 0;
  const ctn_status st =
      ctn_lanczos_which(matvec_cb, &ctx, tmpl.storage_ptr(), n, w, (int)k, nc, (int)maxiter, cvg_crit,
                        (double *)basis.p, (double *)work.p, evals.data(), is_V ? (double *)evecs.p : nullptr, &iters,
                        &nconv, nullptr);
  if (!ctx.err.empty()) throw error(ctx.err);
  check(st, "Lanczos");
  std::vector<UniTensor> out{UniTensor(Tensor::from_vector(evals, {k}, dev), false, 0, {"0"})};
  if (is_V)
    for (cytnx_uint64 j = 0; j < k; ++j) {
      UniTensor v = tmpl.clone();
      check_cuda(cudaMemcpyAsync(v.storage_ptr(), (double *)evecs.p + j * n, n * 8, cudaMemcpyDeviceToDevice, 0),
                 "Lanczos");
      out.push_back(v);
    }
  check_cuda(cudaStreamSynchronize(0), "Lanczos");
  return out;
}

}  // namespace linalg
}  // namespace cytnx
