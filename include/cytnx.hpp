/*
 * cytnx.hpp -- C++ drop-in API (namespace cytnx) for the tensor-network hot path.
 *
 * The classes and free functions below keep the reference's names, argument order and
 * semantics (Cytnx 1.1.1 headers) for what the two-site DMRG path uses, and run every
 * computation through the C ABI of cytnx_b200.h (hand-written sm_100a kernels):
 *
 *   Tensor::permute / permute_ / contiguous / contiguous_   include/Tensor.hpp:718-800
 *   Bond, Symmetry (U1, Zn)                                  include/Bond.hpp:41-71, include/Symmetry.hpp
 *   UniTensor (block-sparse and dense): permute(labels, rowrank), contiguous(_), relabel(s),
 *       contract                                             include/UniTensor.hpp:3791, 4004-4020, 4941
 *   Contract(UniTensor, UniTensor)                           include/UniTensor.hpp:6223
 *   Network::FromString / PutUniTensor / Launch              include/Network.hpp:354, 383, 418
 *   LinOp(type, nx, dtype, device) + virtual matvec          include/LinOp.hpp:68, 163-167
 *   linalg::Tensordot / Matmul / Vectordot / Tridiag         include/linalg.hpp:2435, 2190, 2528, 2575
 *   linalg::Lanczos (method "Gnd" and which "SA/LA/LM")      include/linalg.hpp:2886, 2928
 *
 * Storage lives on a CUDA device (there is no CPU compute path); copies of a Tensor or
 * UniTensor share their storage (the reference's intrusive_ptr semantics) and permute is
 * lazy until contiguous().  Errors throw cytnx::error (a std::logic_error) carrying the C
 * ABI's message; nothing resets the device or exits.  All work is issued on the legacy
 * default stream, in order; a host read (to_vector, item, Norm) synchronises it.
 * Element type of the arithmetic: Type.Double (Tensor permute/contiguous take every dtype).
 */
#ifndef CYTNX_B200_CYTNX_HPP
#define CYTNX_B200_CYTNX_HPP

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "cytnx_b200.h"

namespace cytnx {

typedef double cytnx_double;
typedef float cytnx_float;
typedef int64_t cytnx_int64;
typedef uint64_t cytnx_uint64;
typedef int32_t cytnx_int32;
typedef uint32_t cytnx_uint32;

/* include/cytnx_error.hpp:37-40 */
class error : public std::logic_error {
 public:
  explicit error(const std::string &what) : std::logic_error(what) {}
};

/* dtype ids: include/Type.hpp:177-179 */
struct Type_class {
  static constexpr unsigned int Void = 0, ComplexDouble = 1, ComplexFloat = 2, Double = 3, Float = 4, Int64 = 5,
                                Uint64 = 6, Int32 = 7, Uint32 = 8, Int16 = 9, Uint16 = 10, Bool = 11;
  static std::string getname(unsigned int dtype);
  static size_t typeSize(unsigned int dtype);
};
static constexpr Type_class Type{};

/* device ids: include/Device.hpp (cpu = -1, cuda:i = i) */
struct Device_class {
  static constexpr int cpu = -1, cuda = 0;
};
static constexpr Device_class Device{};

enum bondType : int { BD_KET = -1, BD_BRA = 1, BD_REG = 0, BD_NONE = 0, BD_IN = -1, BD_OUT = 1 };

/* include/Symmetry.hpp: U1 (stype -1) and Zn (stype 0, modulus n) */
class Symmetry {
 public:
  Symmetry() = default;
  static Symmetry U1() { return Symmetry(-1, 1); }
  static Symmetry Zn(int n) { return Symmetry(0, n); }
  int stype() const { return stype_; }
  int n() const { return n_; }
  std::string stype_str() const { return stype_ == -1 ? "U1" : "Z" + std::to_string(n_); }
  bool operator==(const Symmetry &o) const { return stype_ == o.stype_ && n_ == o.n_; }
  bool operator!=(const Symmetry &o) const { return !(*this == o); }

 private:
  Symmetry(int stype, int n) : stype_(stype), n_(n) {}
  int stype_ = -1, n_ = 1;
};

/* include/Bond.hpp:41-71 */
class Bond {
 public:
  Bond() = default;
  Bond(const cytnx_uint64 &dim, const bondType &bd_type = BD_REG);
  Bond(const bondType &bd_type, const std::vector<std::vector<cytnx_int64>> &in_qnums,
       const std::vector<cytnx_uint64> &degs, const std::vector<Symmetry> &in_syms = {});
  cytnx_uint64 dim() const { return dim_; }
  bondType type() const { return type_; }
  cytnx_uint64 Nsym() const { return syms_.size(); }
  cytnx_uint64 Nqnum() const { return degs_.size(); }
  const std::vector<std::vector<cytnx_int64>> &qnums() const { return qnums_; }
  const std::vector<cytnx_uint64> &getDegeneracies() const { return degs_; }
  std::vector<Symmetry> syms() const { return syms_; }
  bool has_qnums() const { return !degs_.empty() && !syms_.empty(); }
  Bond redirect() const;
  Bond &redirect_();
  Bond clone() const { return *this; }
  bool operator==(const Bond &o) const;
  bool operator!=(const Bond &o) const { return !(*this == o); }
  std::string signature() const;  // type, symmetries, charges and degeneracies as text

 private:
  cytnx_uint64 dim_ = 0;
  bondType type_ = BD_REG;
  std::vector<std::vector<cytnx_int64>> qnums_;
  std::vector<cytnx_uint64> degs_;
  std::vector<Symmetry> syms_;
};

namespace detail {
struct DevBuf;  // a device allocation shared by the tensors that view it
struct Layout;  // the blocks of a BlockUniTensor in enumeration order
}  // namespace detail

/* include/Tensor.hpp (storage + shape + the lazy mapper of Tensor_impl) */
class Tensor {
 public:
  Tensor() = default;
  Tensor(const std::vector<cytnx_uint64> &shape, const unsigned int &dtype = Type.Double,
         const int &device = Device.cuda, const bool &init_zero = true);
  /* host -> device copy of `n` elements of `dtype` laid out row-major in `shape` */
  static Tensor from_host(const void *data, const std::vector<cytnx_uint64> &shape,
                          const unsigned int &dtype = Type.Double, const int &device = Device.cuda);
  static Tensor from_vector(const std::vector<double> &v, const std::vector<cytnx_uint64> &shape,
                            const int &device = Device.cuda);
  /* a tensor over the caller's device buffer (row-major, not owned, no copy); the buffer must
   * outlive every tensor that shares it */
  static Tensor from_device(void *ptr, const std::vector<cytnx_uint64> &shape, const unsigned int &dtype = Type.Double,
                            const int &device = Device.cuda);

  std::vector<cytnx_uint64> shape() const { return shape_; }
  unsigned int dtype() const { return dtype_; }
  std::string dtype_str() const { return Type.getname(dtype_); }
  int device() const { return device_; }
  cytnx_uint64 rank() const { return shape_.size(); }
  cytnx_uint64 size() const;  // number of elements
  bool is_contiguous() const;
  const std::vector<cytnx_uint64> &mapper() const { return mapper_; }
  const std::vector<cytnx_uint64> &invmapper() const { return invmapper_; }

  /* Tensor_impl::permute / permute_ (src/backend/Tensor_impl.cpp:38-143): metadata only */
  Tensor permute(const std::vector<cytnx_uint64> &rnks) const;
  Tensor &permute_(const std::vector<cytnx_uint64> &rnks);
  /* Tensor_impl::contiguous / contiguous_ (include/backend/Tensor_impl.hpp:222-325) */
  Tensor contiguous() const;
  Tensor &contiguous_();
  Tensor reshape(const std::vector<cytnx_int64> &new_shape) const;
  Tensor &reshape_(const std::vector<cytnx_int64> &new_shape);
  Tensor clone() const;

  /* device -> host copy of the elements in logical row-major order */
  std::vector<double> to_vector() const;                // Double only
  void to_host(void *dst) const;                        // any dtype, size() elements
  double item() const;                                  // one-element Double tensor
  void *device_ptr() const;                             // first element of the storage (physical order)

 private:
  friend class UniTensor;
  std::shared_ptr<detail::DevBuf> buf_;
  cytnx_uint64 offset_ = 0;  // element offset of this tensor inside buf_
  std::vector<cytnx_uint64> shape_, mapper_, invmapper_;
  unsigned int dtype_ = Type.Double;
  int device_ = Device.cuda;
};

/* include/UniTensor.hpp: block-sparse (BlockUniTensor) and dense (DenseUniTensor) forms */
class UniTensor {
 public:
  UniTensor() = default;
  /* block form when the bonds carry quantum numbers, dense otherwise */
  UniTensor(const std::vector<Bond> &bonds, const std::vector<std::string> &in_labels = {},
            const cytnx_int64 &rowrank = -1, const unsigned int &dtype = Type.Double,
            const int &device = Device.cuda, const bool &is_diag = false, const std::string &name = "");
  /* dense form around a Tensor (shares its storage) */
  explicit UniTensor(const Tensor &in_tensor, const bool &is_diag = false, const cytnx_int64 &rowrank = -1,
                     const std::vector<std::string> &in_labels = {}, const std::string &name = "");

  bool is_blockform() const { return block_; }
  cytnx_uint64 rank() const { return bonds_.size(); }
  cytnx_int64 rowrank() const { return rowrank_; }
  std::vector<std::string> labels() const { return labels_; }
  const std::vector<Bond> &bonds() const { return bonds_; }
  std::vector<cytnx_uint64> shape() const;
  unsigned int dtype() const { return Type.Double; }
  int device() const { return device_; }
  std::string name() const { return name_; }
  cytnx_uint64 Nblocks() const;
  bool is_contiguous() const;
  /* logical qnum-index tuple of every block (BlockUniTensor::get_itoi) */
  std::vector<std::vector<cytnx_uint64>> get_itoi() const;

  UniTensor &set_name(const std::string &name) {
    name_ = name;
    return *this;
  }
  UniTensor &set_rowrank_(const cytnx_uint64 &new_rowrank);
  UniTensor set_rowrank(const cytnx_uint64 &new_rowrank) const;
  UniTensor &set_labels(const std::vector<std::string> &new_labels);
  UniTensor relabel(const std::vector<std::string> &new_labels) const;
  UniTensor relabels(const std::vector<std::string> &new_labels) const { return relabel(new_labels); }
  UniTensor &relabel_(const std::vector<std::string> &new_labels);
  UniTensor relabel(const std::string &old_label, const std::string &new_label) const;
  UniTensor &relabel_(const std::string &old_label, const std::string &new_label);

  /* BlockUniTensor::permute (src/BlockUniTensor.cpp:588-708): bonds, labels, qnum tuples, lazy data */
  UniTensor permute(const std::vector<cytnx_int64> &mapper, const cytnx_int64 &rowrank = -1) const;
  UniTensor permute(const std::vector<std::string> &mapper, const cytnx_int64 &rowrank = -1) const;
  UniTensor &permute_(const std::vector<cytnx_int64> &mapper, const cytnx_int64 &rowrank = -1);
  UniTensor &permute_(const std::vector<std::string> &mapper, const cytnx_int64 &rowrank = -1);
  UniTensor contiguous() const;
  void contiguous_();

  /* a copy of block idx (dense: the one block) in logical leg order */
  Tensor get_block(const cytnx_uint64 &idx = 0) const;
  /* the block with the given qnum indices; throws if it is not allowed */
  Tensor get_block(const std::vector<cytnx_int64> &qidx) const;
  void put_block(const Tensor &in, const cytnx_uint64 &idx = 0);
  void put_block(const Tensor &in, const std::vector<cytnx_int64> &qidx);

  /* BlockUniTensor::contract (src/BlockUniTensor.cpp:777-1235) */
  UniTensor contract(const UniTensor &rhs, const bool &mv_elem_self = false, const bool &mv_elem_rhs = false) const;
  Tensor Norm() const;  // one-element Double tensor on the device
  UniTensor Conj() const { return *this; }  // real data
  UniTensor Transpose() const;               // BlockUniTensor::Transpose_ (src/BlockUniTensor.cpp:1237-1245)
  UniTensor Dagger() const { return Transpose(); }
  UniTensor clone() const;

  /* same structure, elementwise (contiguous storage of both) */
  UniTensor operator+(const UniTensor &rhs) const;
  UniTensor operator-(const UniTensor &rhs) const;
  UniTensor operator*(const double &a) const;
  UniTensor operator/(const double &a) const;
  UniTensor &operator+=(const UniTensor &rhs);
  UniTensor &operator-=(const UniTensor &rhs);
  UniTensor &operator*=(const double &a);
  UniTensor &operator/=(const double &a);

  /* the storage as one flat vector of every block back to back (block order, each block
   * row-major in logical leg order after contiguous()) */
  std::vector<double> to_vector() const;
  void from_vector(const std::vector<double> &flat);
  cytnx_uint64 storage_size() const;  // elements
  double *storage_ptr() const;        // device pointer (physical order)
  /* a tensor with this one's structure over the caller's device buffer (no copy, not owned) */
  UniTensor view_of(double *device_flat) const;

 private:
  friend UniTensor Contract(const UniTensor &, const UniTensor &, const bool &, const bool &);
  friend class Network;
  bool block_ = false;
  std::vector<Bond> bonds_;
  std::vector<std::string> labels_;
  cytnx_int64 rowrank_ = 0;
  bool is_diag_ = false;
  std::string name_;
  int device_ = Device.cuda;
  std::shared_ptr<const detail::Layout> layout_;  // block form: blocks of the stored leg order
  std::vector<cytnx_uint64> mapper_;               // block form: lazy permutation (logical -> stored)
  std::shared_ptr<detail::DevBuf> buf_;            // block form: all blocks back to back
  Tensor dense_;                                   // dense form
  std::vector<Bond> stored_bonds() const;
  void check_same_structure(const UniTensor &o, const char *where) const;
};

UniTensor Contract(const UniTensor &inL, const UniTensor &inR, const bool &cacheL = false,
                   const bool &cacheR = false);

/* include/LinOp.hpp:68-167: subclass and override matvec */
class LinOp {
 public:
  LinOp(const std::string &type, const cytnx_uint64 &nx, const int &dtype = Type.Double,
        const int &device = Device.cpu);
  virtual ~LinOp() = default;
  int device() const { return device_; }
  int dtype() const { return dtype_; }
  cytnx_uint64 nx() const { return nx_; }
  virtual Tensor matvec(const Tensor &Tin);
  virtual UniTensor matvec(const UniTensor &Tin);

 private:
  std::string type_;
  cytnx_uint64 nx_ = 0;
  int dtype_ = Type.Double, device_ = Device.cpu;
};

/* include/Network.hpp (RegularNetwork): FromString lines "name: l1,l2;l3", "TOUT: a;b",
 * optional "ORDER: ((A,B),C)"; default tree = left fold in declaration order */
class Network {
 public:
  Network() = default;
  explicit Network(const std::string &fname) { Fromfile(fname); }
  void Fromfile(const std::string &fname);
  void FromString(const std::vector<std::string> &contents);
  void PutUniTensor(const std::string &name, const UniTensor &utensor,
                    const std::vector<std::string> &label_order = {});
  void PutUniTensor(const cytnx_uint64 &idx, const UniTensor &utensor,
                    const std::vector<std::string> &label_order = {});
  void PutUniTensors(const std::vector<std::string> &names, const std::vector<UniTensor> &utensors);
  void RmUniTensor(const std::string &name);
  void setOrder(const bool &optimal, const std::string &contract_order);
  std::string getOrder() const;
  UniTensor Launch();

 private:
  std::vector<std::string> names_;
  std::vector<std::vector<std::string>> labels_;
  std::map<std::string, UniTensor> tensors_;
  std::vector<std::string> tout_;
  cytnx_int64 tout_rowrank_ = 0;
  std::string order_;
  bool optimal_ = false;
};

namespace linalg {
/* include/linalg.hpp:2435 */
Tensor Tensordot(const Tensor &Tl, const Tensor &Tr, const std::vector<cytnx_uint64> &idxl,
                 const std::vector<cytnx_uint64> &idxr, const bool &cacheL = false, const bool &cacheR = false);
/* include/linalg.hpp:2190 (rank-2 x rank-2) */
Tensor Matmul(const Tensor &Tl, const Tensor &Tr);
/* include/linalg.hpp:2528 (rank-1, real) */
Tensor Vectordot(const Tensor &Tl, const Tensor &Tr, const bool &is_conj = false);
/* include/linalg.hpp:2575: [eigenvalues, eigenvectors (rows if is_row)] */
std::vector<Tensor> Tridiag(const Tensor &Diag, const Tensor &Sub_diag, const bool &is_V = true,
                            const bool &is_row = false, bool throw_excp = false);
/* include/linalg.hpp:2928 (method "Gnd": Lanczos_Gnd_Ut / Lanczos_Gnd):
 * returns {eigenvalue (rank-1 UniTensor of one element), eigenvector (Tin's structure)} */
std::vector<UniTensor> Lanczos(LinOp *Hop, const UniTensor &Tin = UniTensor(), const std::string method = "Gnd",
                               const double &CvgCrit = 1.0e-14, const unsigned int &Maxiter = 10000,
                               const cytnx_uint64 &k = 1, const bool &is_V = true, const bool &is_row = false,
                               const cytnx_uint32 &max_krydim = 4, const bool &verbose = false);
std::vector<Tensor> Lanczos(LinOp *Hop, const Tensor &Tin, const std::string method = "Gnd",
                            const double &CvgCrit = 1.0e-14, const unsigned int &Maxiter = 10000,
                            const cytnx_uint64 &k = 1, const bool &is_V = true, const bool &is_row = false,
                            const cytnx_uint32 &max_krydim = 4, const bool &verbose = false);
/* include/linalg.hpp:2886 (which = "SA", "LA", "LM"): {eigenvalues, eigenvectors...} */
std::vector<UniTensor> Lanczos(LinOp *Hop, const UniTensor &Tin, const std::string which,
                               const cytnx_uint64 &maxiter, const cytnx_double &cvg_crit = 0,
                               const cytnx_uint64 &k = 1, const bool &is_V = true, const cytnx_int32 &ncv = 0,
                               const bool &verbose = false);
}  // namespace linalg

}  // namespace cytnx

#endif
