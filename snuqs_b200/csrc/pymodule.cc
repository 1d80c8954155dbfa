// pybind11 module `snuqs_b200._C`: the reference's `braket.snuqs._C` surface
// (src/braket/snuqs/csrc/pymodule.cc:66-210) -- same submodules, class names,
// constructor signatures, keyword arguments and buffer protocols -- on top of
// the C ABI in include/snuqs_b200.h.  Nothing here computes on the state:
// every state operation goes through an sq_* call.
//
// Differences a caller can observe, all deliberate:
//   * functionals.apply queues the gate; the queue runs as fused sweeps at
//     the next sync()/cpu()/copy()/flush (the reference launches one kernel
//     per call and ignores `stream`, functionals.cc:15-28).
//   * ctrl_modifiers and power are honoured (the reference stores them and
//     never applies them, operation.cc:96-109); power may be negative or
//     fractional (the reference binds it as size_t).
//   * errors raise RuntimeError/ValueError instead of exiting the process
//     (utils_cuda.h:8-16).
//   * a CPU StateVector is a host buffer only: applying gates to it raises
//     (the engine has no CPU path).
#include <pybind11/complex.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cmath>
#include <complex>
#include <cstring>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <unistd.h>

#include "../../include/snuqs_b200.h"

namespace py = pybind11;
using cplx = std::complex<double>;

static void check(int status) {
  if (status != SQ_OK) {
    std::string msg = sq_last_error();
    if (status == SQ_ERR_INVALID) throw py::value_error(msg);
    throw std::runtime_error(msg);
  }
}

enum class DeviceType { CPU = 0, CUDA = 1, STORAGE = 2 };

// ---------------------------------------------------------------------------
// Stream / Event (stream.cc:6-34, event.cc:5-26)
// ---------------------------------------------------------------------------
class Event;
class Stream {
 public:
  explicit Stream(void *s, bool owns = false) : s_(s), owns_(owns) {}
  ~Stream() {
    if (owns_ && s_) sq_stream_destroy(s_);
  }
  void *get() const { return s_; }
  void synchronize() { check(sq_stream_synchronize(s_)); }
  void wait_event(std::shared_ptr<Event> e);
  static std::shared_ptr<Stream> create() {
    void *s = nullptr;
    check(sq_stream_create(&s, 0));
    return std::make_shared<Stream>(s, true);
  }
  static std::shared_ptr<Stream> create_nonblocking() {
    void *s = nullptr;
    check(sq_stream_create(&s, 1));
    return std::make_shared<Stream>(s, true);
  }

 private:
  void *s_;
  bool owns_;
};

class Event {
 public:
  explicit Event(void *e, bool owns = false) : e_(e), owns_(owns) {}
  ~Event() {
    if (owns_ && e_) sq_event_destroy(e_);
  }
  void *get() const { return e_; }
  void record(std::shared_ptr<Stream> s) {
    check(sq_event_record(e_, s ? s->get() : nullptr));
  }
  void synchronize() { check(sq_event_synchronize(e_)); }
  static std::shared_ptr<Event> create() {
    void *e = nullptr;
    check(sq_event_create(&e));
    return std::make_shared<Event>(e, true);
  }

 private:
  void *e_;
  bool owns_;
};

void Stream::wait_event(std::shared_ptr<Event> e) {
  check(sq_stream_wait_event(s_, e->get()));
}

static void *stream_ptr(const std::shared_ptr<Stream> &s) { return s ? s->get() : nullptr; }

// ---------------------------------------------------------------------------
// Operations (operation.h:8-90, gate_operations.h)
// ---------------------------------------------------------------------------
class Operation {
 public:
  explicit Operation(const std::vector<size_t> &targets) : targets_(targets) {}
  virtual ~Operation() = default;
  std::vector<size_t> get_targets() const { return targets_; }
  void set_targets(const std::vector<size_t> &t) { targets_ = t; }
  std::vector<size_t> targets_;
};

static const char *kGateNames[] = {
    "Identity", "Hadamard", "PauliX", "PauliY", "PauliZ", "CX", "CY", "CZ", "S", "Si", "T",
    "Ti", "V", "Vi", "PhaseShift", "CPhaseShift", "CPhaseShift00", "CPhaseShift01",
    "CPhaseShift10", "RotX", "RotY", "RotZ", "Swap", "ISwap", "PSwap", "XY", "XX", "YY", "ZZ",
    "CCNot", "CSwap", "U", "GPhase", "SwapA2A", "ECR", "CV", "PRx"};
constexpr int kUnitaryType = SQ_GATE_COUNT;  // GateOperationType.Unitary
// Angles each named gate takes (gate_operations.h; U has 3, PRx 2).
static const int kGateAngles[SQ_GATE_COUNT] = {
    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 1, 1, 1, 1, 1,
    0, 0, 3, 1, 0, 0, 0, 2};
enum class GateOperationType : int {};

// Square matrix helpers for the power modifier.
static std::vector<cplx> matmul(const std::vector<cplx> &a, const std::vector<cplx> &b, int d) {
  std::vector<cplx> c(size_t(d) * d, cplx(0, 0));
  for (int i = 0; i < d; ++i)
    for (int k = 0; k < d; ++k)
      for (int j = 0; j < d; ++j) c[size_t(i) * d + j] += a[size_t(i) * d + k] * b[size_t(k) * d + j];
  return c;
}
static std::vector<cplx> dagger(const std::vector<cplx> &a, int d) {
  std::vector<cplx> c(size_t(d) * d);
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) c[size_t(j) * d + i] = std::conj(a[size_t(i) * d + j]);
  return c;
}

class GateOperation : public Operation {
 public:
  GateOperation(int type, const std::vector<size_t> &targets, const std::vector<double> &angles,
                const std::vector<size_t> &ctrl_modifiers, double power)
      : Operation(targets), type_(type), angles_(angles), ctrl_(ctrl_modifiers), power_(power) {
    if (type_ != kUnitaryType) {
      std::vector<double> a = angles_;
      a.resize(3, 0.0);
      uint32_t k = 0;
      base_.assign(64, cplx(0, 0));
      check(sq_gate_matrix(type_, a.data(), uint32_t(angles_.size()),
                           reinterpret_cast<double *>(base_.data()), &k));
      base_.resize(size_t(1) << (2 * k));
      base_k_ = int(k);
    }
    finalize();
  }
  // Unitary(targets, matrix): the reference's Python Unitary
  // (src/braket/snuqs/gate_operations.py:23-39) cannot be constructed (it
  // passes keywords the pybind ctor rejects); this one takes the matrix.
  GateOperation(const std::vector<size_t> &targets, py::array_t<cplx> matrix,
                const std::vector<size_t> &ctrl_modifiers, double power)
      : Operation(targets), type_(kUnitaryType), ctrl_(ctrl_modifiers), power_(power) {
    auto m = matrix.unchecked<2>();
    const size_t d = size_t(m.shape(0));
    if (m.shape(1) != ssize_t(d) || (d & (d - 1)) || d == 0)
      throw py::value_error("Unitary matrix must be square with a power-of-two size");
    base_k_ = 0;
    while ((size_t(1) << base_k_) < d) ++base_k_;
    base_.resize(d * d);
    for (size_t i = 0; i < d; ++i)
      for (size_t j = 0; j < d; ++j) base_[i * d + j] = m(i, j);
    finalize();
  }
  virtual ~GateOperation() = default;

  // Effective matrix over all targets: controlled(base^power).
  void finalize() {
    const size_t nc = ctrl_.size();
    if (targets_.size() != nc + size_t(base_k_))
      throw py::value_error("gate " + name() + " expects " + std::to_string(nc + base_k_) +
                            " targets (" + std::to_string(nc) + " controls + " +
                            std::to_string(base_k_) + "), got " +
                            std::to_string(targets_.size()));
    const int d = 1 << base_k_;
    powered_ = base_;
    if (power_ != 1.0) {
      const double r = std::round(power_);
      if (std::fabs(power_ - r) > 0)
        throw py::value_error("fractional gate powers are handled by the Python front end");
      std::vector<cplx> b = r < 0 ? dagger(base_, d) : base_;
      std::vector<cplx> acc(size_t(d) * d, cplx(0, 0));
      for (int i = 0; i < d; ++i) acc[size_t(i) * d + i] = 1.0;
      for (long e = 0; e < std::labs(long(r)); ++e) acc = matmul(acc, b, d);
      powered_ = acc;
    }
    const int kk = int(targets_.size());
    const size_t D = size_t(1) << kk;
    full_.assign(D * D, cplx(0, 0));
    // Control qubits are the leading (most significant) targets.
    size_t cidx = 0;
    for (size_t c = 0; c < nc; ++c) cidx = (cidx << 1) | (ctrl_[c] ? 1 : 0);
    for (size_t r = 0; r < D; ++r) {
      const size_t rc = r >> base_k_;
      if (rc != cidx) {
        full_[r * D + r] = 1.0;
        continue;
      }
      for (size_t c = 0; c < size_t(d); ++c)
        full_[r * D + ((cidx << base_k_) | c)] = powered_[(r & (d - 1)) * d + c];
    }
  }

  std::string name() const {
    return type_ == kUnitaryType ? "Unitary" : (type_ >= 0 && type_ < SQ_GATE_COUNT ? kGateNames[type_] : "?");
  }
  std::string formatted_string() const {
    std::stringstream ss;
    ss << name();
    if (!angles_.empty()) {
      ss << "(";
      for (size_t i = 0; i < angles_.size(); ++i) ss << angles_[i] << (i + 1 < angles_.size() ? ", " : "");
      ss << ")";
    }
    ss << " {";
    for (size_t i = 0; i < targets_.size(); ++i) ss << targets_[i] << (i + 1 < targets_.size() ? ", " : "");
    ss << "}";
    return ss.str();
  }
  bool operator==(const GateOperation &o) const {
    return type_ == o.type_ && targets_ == o.targets_ && angles_ == o.angles_ && ctrl_ == o.ctrl_ &&
           power_ == o.power_ && (type_ != kUnitaryType || base_ == o.base_);
  }
  size_t dim_() const { return size_t(1) << targets_.size(); }
  py::buffer_info buffer() {
    const ssize_t D = ssize_t(dim_());
    return py::buffer_info(full_.data(), sizeof(cplx), py::format_descriptor<cplx>::format(), 2,
                           {D, D}, {ssize_t(D * sizeof(cplx)), ssize_t(sizeof(cplx))});
  }

  int type_;
  std::vector<double> angles_;
  std::vector<size_t> ctrl_;
  double power_;
  int base_k_ = 0;
  std::vector<cplx> base_, powered_, full_;
};

// ---------------------------------------------------------------------------
// StateVector (state_vector.h:10-41)
// ---------------------------------------------------------------------------
struct HostBuffer {
  void *p = nullptr;
  bool pinned = false;
  explicit HostBuffer(size_t bytes, bool pin) : pinned(pin) {
    if (pin) {
      check(sq_host_alloc(&p, bytes));
    } else {
      p = std::aligned_alloc(4096, (bytes + 4095) & ~size_t(4095));
      if (!p) throw std::bad_alloc();
    }
  }
  ~HostBuffer() {
    if (pinned) sq_host_free(p);
    else std::free(p);
  }
};

struct DeviceState {
  sq_state *s = nullptr;
  ~DeviceState() {
    if (s) sq_state_destroy(s);
  }
};

class StateVector : public std::enable_shared_from_this<StateVector> {
 public:
  StateVector(size_t n) : StateVector(DeviceType::CPU, n, false, SQ_C128) {}
  StateVector(size_t n, bool pinned) : StateVector(DeviceType::CPU, n, pinned, SQ_C128) {}
  StateVector(DeviceType dev, size_t n) : StateVector(dev, n, false, SQ_C128) {}
  StateVector(DeviceType dev, size_t n, bool pinned, int dtype) : dev_(dev), n_(n), dtype_(dtype) {
    if (dev == DeviceType::STORAGE)
      throw std::runtime_error("STORAGE state vectors (NVMe offload) are not supported by this engine");
    if (dev == DeviceType::CUDA) {
      ds_ = std::make_shared<DeviceState>();
      check(sq_state_create(uint32_t(n), dtype, &ds_->s));
    } else {
      hb_ = std::make_shared<HostBuffer>(bytes(), pinned);
      host_ = hb_->p;
    }
  }
  // Host view sharing an owner (slice()).
  StateVector(size_t n, int dtype, std::shared_ptr<HostBuffer> owner, void *p)
      : dev_(DeviceType::CPU), n_(n), dtype_(dtype), hb_(std::move(owner)), host_(p) {}

  size_t amp_bytes() const { return dtype_ == SQ_C64 ? 8 : 16; }
  size_t bytes() const { return (size_t(1) << n_) * amp_bytes(); }
  sq_state *dev() const {
    if (dev_ != DeviceType::CUDA) throw std::runtime_error("state vector is not on CUDA");
    return ds_->s;
  }

  std::shared_ptr<StateVector> cpu(std::shared_ptr<Stream> stream) {
    if (dev_ == DeviceType::CPU) return shared_from_this();
    auto out = std::make_shared<StateVector>(DeviceType::CPU, n_, false, dtype_);
    {
      py::gil_scoped_release nogil;
      check(sq_copy_to_host(ds_->s, out->host_, stream_ptr(stream)));
      check(sq_stream_synchronize(stream_ptr(stream)));
    }
    return out;
  }
  std::shared_ptr<StateVector> cuda(std::shared_ptr<Stream> stream) {
    if (dev_ == DeviceType::CUDA) return shared_from_this();
    auto out = std::make_shared<StateVector>(DeviceType::CUDA, n_, false, dtype_);
    py::gil_scoped_release nogil;
    check(sq_copy_from_host(out->ds_->s, host_, stream_ptr(stream)));
    check(sq_stream_synchronize(stream_ptr(stream)));
    return out;
  }
  void copy(StateVector &other, std::shared_ptr<Stream> stream) {
    if (other.n_ != n_ || other.dtype_ != dtype_)
      throw py::value_error("copy between state vectors of different size or precision");
    py::gil_scoped_release nogil;
    void *st = stream_ptr(stream);
    if (dev_ == DeviceType::CUDA && other.dev_ == DeviceType::CUDA) {
      check(sq_copy_state(ds_->s, other.ds_->s, st));
    } else if (dev_ == DeviceType::CUDA) {
      check(sq_copy_from_host(ds_->s, other.host_, st));
    } else if (other.dev_ == DeviceType::CUDA) {
      check(sq_copy_to_host(other.ds_->s, host_, st));
    } else {
      std::memcpy(host_, other.host_, bytes());
      return;
    }
    check(sq_stream_synchronize(st));
  }
  std::shared_ptr<StateVector> slice(size_t nsliced, size_t index) {
    if (dev_ != DeviceType::CPU)
      throw std::runtime_error("slicing a device state is not supported (no state slicing in this engine)");
    if (nsliced > n_ || ((index + 1) << nsliced) > (size_t(1) << n_))
      throw py::value_error("slice out of range");
    return std::make_shared<StateVector>(nsliced, dtype_, hb_,
                                         static_cast<char *>(host_) + (index << nsliced) * amp_bytes());
  }
  void sync() {
    if (dev_ != DeviceType::CUDA) return;
    py::gil_scoped_release nogil;
    check(sq_flush(ds_->s, nullptr));
    check(sq_device_synchronize());
  }
  std::string formatted_string() const {
    std::stringstream ss;
    ss << "StateVector<" << n_ << " qubits, device: "
       << (dev_ == DeviceType::CPU ? "CPU" : dev_ == DeviceType::CUDA ? "CUDA" : "STORAGE")
       << (dtype_ == SQ_C64 ? ", complex64" : "") << ">";
    return ss.str();
  }
  py::buffer_info buffer() {
    if (dev_ != DeviceType::CPU)
      throw py::buffer_error("a CUDA state vector has no host buffer; call .cpu() first");
    if (dtype_ == SQ_C64)
      return py::buffer_info(host_, 8, py::format_descriptor<std::complex<float>>::format(), 1,
                             {ssize_t(size_t(1) << n_)}, {ssize_t(8)});
    return py::buffer_info(host_, sizeof(cplx), py::format_descriptor<cplx>::format(), 1,
                           {ssize_t(size_t(1) << n_)}, {ssize_t(sizeof(cplx))});
  }

  DeviceType dev_;
  size_t n_;
  int dtype_;
  std::shared_ptr<DeviceState> ds_;
  std::shared_ptr<HostBuffer> hb_;
  void *host_ = nullptr;
};

// ---------------------------------------------------------------------------
// functionals (functionals.h:10-15)
// ---------------------------------------------------------------------------
static void apply(StateVector &sv, GateOperation &op, size_t num_qubits, std::vector<size_t> targets,
                  std::shared_ptr<Stream> stream) {
  if (sv.dev_ != DeviceType::CUDA)
    throw std::runtime_error(
        "functionals.apply: this engine simulates CUDA state vectors only "
        "(create the state with DeviceType.CUDA)");
  if (num_qubits != sv.n_)
    throw py::value_error("num_qubits does not match the state vector");
  if (targets.size() != op.targets_.size())
    throw py::value_error("target count does not match the gate");
  const size_t nc = op.ctrl_.size();
  std::vector<uint32_t> ctrl(targets.begin(), targets.begin() + nc);
  std::vector<uint32_t> tq(targets.begin() + nc, targets.end());
  std::vector<uint8_t> cv(nc);
  for (size_t i = 0; i < nc; ++i) cv[i] = op.ctrl_[i] ? 1 : 0;
  check(sq_apply_controlled_matrix(sv.dev(), reinterpret_cast<const double *>(op.powered_.data()),
                                   tq.data(), uint32_t(tq.size()), ctrl.data(), cv.data(),
                                   uint32_t(nc), stream_ptr(stream)));
}

static void initialize_zero(StateVector &sv, std::shared_ptr<Stream> stream) {
  if (sv.dev_ == DeviceType::CUDA) {
    check(sq_init_zero(sv.dev(), stream_ptr(stream)));
  } else {
    std::memset(sv.host_, 0, sv.bytes());
  }
}

static void initialize_basis_z(StateVector &sv, std::shared_ptr<Stream> stream) {
  if (sv.dev_ == DeviceType::CUDA) {
    check(sq_init_basis(sv.dev(), 0, stream_ptr(stream)));
  } else {
    std::memset(sv.host_, 0, sv.bytes());
    if (sv.dtype_ == SQ_C64) static_cast<std::complex<float> *>(sv.host_)[0] = 1.0f;
    else static_cast<cplx *>(sv.host_)[0] = 1.0;
  }
}

// Each named gate is its own class deriving from GateOperation, with the
// reference's constructor signatures (GATEOP / GATEOP1 / GATEOP3,
// pymodule.cc:20-64); PRx takes two angles.
template <int ID>
struct NamedGate : GateOperation {
  NamedGate(const std::vector<size_t> &t, const std::vector<double> &a,
            const std::vector<size_t> &c, double p)
      : GateOperation(ID, t, a, c, p) {}
};
struct Unitary : GateOperation {
  Unitary(const std::vector<size_t> &t, py::array_t<cplx> m, const std::vector<size_t> &c, double p)
      : GateOperation(t, m, c, p) {}
};

template <int ID>
static void def_gate(py::module_ &mod, const char *name) {
  auto cls = py::class_<NamedGate<ID>, GateOperation, std::shared_ptr<NamedGate<ID>>>(
      mod, name, py::buffer_protocol());
  cls.def_buffer([](NamedGate<ID> &g) { return g.buffer(); });
  const int na = kGateAngles[ID];
  using V = std::vector<size_t>;
  if (na == 3) {
    cls.def(py::init([](const V &t, double a1, double a2, double a3, const V &c, double p) {
              return std::make_shared<NamedGate<ID>>(t, std::vector<double>{a1, a2, a3}, c, p);
            }),
            py::arg("targets"), py::arg("angle_1"), py::arg("angle_2"), py::arg("angle_3"),
            py::kw_only(), py::arg("ctrl_modifiers") = V(), py::arg("power") = 1.0);
  } else if (na == 2) {
    cls.def(py::init([](const V &t, double a1, double a2, const V &c, double p) {
              return std::make_shared<NamedGate<ID>>(t, std::vector<double>{a1, a2}, c, p);
            }),
            py::arg("targets"), py::arg("angle_1"), py::arg("angle_2"), py::kw_only(),
            py::arg("ctrl_modifiers") = V(), py::arg("power") = 1.0);
  } else if (na == 1) {
    cls.def(py::init([](const V &t, double a, const V &c, double p) {
              return std::make_shared<NamedGate<ID>>(t, std::vector<double>{a}, c, p);
            }),
            py::arg("targets"), py::arg("angle"), py::kw_only(), py::arg("ctrl_modifiers") = V(),
            py::arg("power") = 1.0);
  } else {
    cls.def(py::init([](const V &t, const V &c, double p) {
              return std::make_shared<NamedGate<ID>>(t, std::vector<double>{}, c, p);
            }),
            py::arg("targets"), py::kw_only(), py::arg("ctrl_modifiers") = V(),
            py::arg("power") = 1.0);
  }
}

PYBIND11_MODULE(_C, m) {
  m.doc() = "snuqs_b200: B200 state-vector engine with the SnuQS _C interface.";

  py::enum_<DeviceType>(m, "DeviceType")
      .value("CPU", DeviceType::CPU)
      .value("CUDA", DeviceType::CUDA)
      .value("STORAGE", DeviceType::STORAGE)
      .export_values();

  auto m_operation = m.def_submodule("operation");
  py::class_<Operation, std::shared_ptr<Operation>>(m_operation, "Operation")
      .def(py::init<const std::vector<size_t> &>())
      .def_property("targets", &Operation::get_targets, &Operation::set_targets);

  auto gtype = py::enum_<GateOperationType>(m_operation, "GateOperationType");
  for (int i = 0; i < SQ_GATE_COUNT; ++i) gtype.value(kGateNames[i], GateOperationType(i));
  gtype.value("Unitary", GateOperationType(kUnitaryType));

  py::class_<GateOperation, Operation, std::shared_ptr<GateOperation>>(
      m_operation, "GateOperation", py::buffer_protocol())
      .def(py::init([](GateOperationType t, const std::vector<size_t> &tg,
                       const std::vector<double> &a, const std::vector<size_t> &c, double p) {
             return std::make_shared<GateOperation>(int(t), tg, a, c, p);
           }),
           py::arg("type"), py::arg("targets"), py::arg("angles") = std::vector<double>(),
           py::arg("ctrl_modifiers") = std::vector<size_t>(), py::arg("power") = 1.0)
      .def_buffer(&GateOperation::buffer)
      .def("sliceable", [](const GateOperation &) { return false; })
      .def("slice", [](const GateOperation &g, size_t) { return std::make_shared<GateOperation>(g); })
      .def("__repr__", &GateOperation::formatted_string)
      .def("__eq__", &GateOperation::operator==)
      .def_property_readonly("name", &GateOperation::name)
      .def_property_readonly("type", [](const GateOperation &g) { return g.type_; })
      .def_property_readonly("angles", [](const GateOperation &g) { return g.angles_; })
      .def_property_readonly("ctrl_modifiers", [](const GateOperation &g) { return g.ctrl_; })
      .def_property_readonly("power", [](const GateOperation &g) { return g.power_; })
      .def_property_readonly("base_matrix", [](const GateOperation &g) {
        const ssize_t d = ssize_t(1) << g.base_k_;
        py::array_t<cplx> a({d, d});
        std::memcpy(a.mutable_data(), g.powered_.data(), size_t(d * d) * sizeof(cplx));
        return a;
      });

  auto m_gate_operations = m_operation.def_submodule("gate_operations");
#define SQ_DEF(ID) def_gate<ID>(m_gate_operations, kGateNames[ID]);
  SQ_DEF(0) SQ_DEF(1) SQ_DEF(2) SQ_DEF(3) SQ_DEF(4) SQ_DEF(5) SQ_DEF(6) SQ_DEF(7) SQ_DEF(8)
  SQ_DEF(9) SQ_DEF(10) SQ_DEF(11) SQ_DEF(12) SQ_DEF(13) SQ_DEF(14) SQ_DEF(15) SQ_DEF(16)
  SQ_DEF(17) SQ_DEF(18) SQ_DEF(19) SQ_DEF(20) SQ_DEF(21) SQ_DEF(22) SQ_DEF(23) SQ_DEF(24)
  SQ_DEF(25) SQ_DEF(26) SQ_DEF(27) SQ_DEF(28) SQ_DEF(29) SQ_DEF(30) SQ_DEF(31) SQ_DEF(32)
  SQ_DEF(34) SQ_DEF(35) SQ_DEF(36)
#undef SQ_DEF
  py::class_<Unitary, GateOperation, std::shared_ptr<Unitary>>(m_gate_operations, "Unitary",
                                                               py::buffer_protocol())
      .def_buffer([](Unitary &g) { return g.buffer(); })
      .def(py::init<const std::vector<size_t> &, py::array_t<cplx>, const std::vector<size_t> &,
                    double>(),
           py::arg("targets"), py::arg("matrix"), py::kw_only(),
           py::arg("ctrl_modifiers") = std::vector<size_t>(), py::arg("power") = 1.0);
  m.attr("_gate_names") = py::cast(std::vector<std::string>(std::begin(kGateNames), std::end(kGateNames)));

  // Stream
  auto m_stream = m.def_submodule("stream");
  py::class_<Stream, std::shared_ptr<Stream>>(m_stream, "Stream")
      .def(py::init([](uintptr_t p) { return std::make_shared<Stream>(reinterpret_cast<void *>(p)); }))
      .def("get", [](const Stream &s) { return reinterpret_cast<uintptr_t>(s.get()); })
      .def("synchronize", &Stream::synchronize)
      .def("wait_event", &Stream::wait_event)
      .def_static("create", &Stream::create)
      .def_static("create_nonblocking", &Stream::create_nonblocking);

  // Event
  auto m_event = m.def_submodule("event");
  py::class_<Event, std::shared_ptr<Event>>(m_event, "Event")
      .def(py::init([](uintptr_t p) { return std::make_shared<Event>(reinterpret_cast<void *>(p)); }))
      .def("get", [](const Event &e) { return reinterpret_cast<uintptr_t>(e.get()); })
      .def("record", &Event::record)
      .def("synchronize", &Event::synchronize)
      .def_static("create", &Event::create);

  // Functionals
  auto m_functionals = m.def_submodule("functionals");
  m_functionals.def("apply", &apply, py::arg("state_vector"), py::arg("op"), py::arg("num_qubits"),
                    py::arg("targets"), py::kw_only(), py::arg("stream") = nullptr);
  m_functionals.def("initialize_zero", &initialize_zero, py::arg("state_vector"), py::kw_only(),
                    py::arg("stream") = nullptr);
  m_functionals.def("initialize_basis_z", &initialize_basis_z, py::arg("state_vector"),
                    py::kw_only(), py::arg("stream") = nullptr);
  m_functionals.def(
      "flush",
      [](StateVector &sv, std::shared_ptr<Stream> stream) {
        py::gil_scoped_release nogil;
        check(sq_flush(sv.dev(), stream_ptr(stream)));
      },
      py::arg("state_vector"), py::kw_only(), py::arg("stream") = nullptr);
  m_functionals.def(
      "probabilities",
      [](StateVector &sv, uintptr_t out_device, std::shared_ptr<Stream> stream) {
        py::gil_scoped_release nogil;
        check(sq_probabilities(sv.dev(), reinterpret_cast<double *>(out_device), stream_ptr(stream)));
      },
      py::arg("state_vector"), py::arg("out_device_ptr"), py::kw_only(),
      py::arg("stream") = nullptr);
  m_functionals.def(
      "expectation",
      [](StateVector &sv, const std::vector<std::string> &paulis, const std::vector<double> &weights,
         std::shared_ptr<Stream> stream) {
        if (paulis.size() != weights.size()) throw py::value_error("one weight per Pauli string");
        std::string flat;
        for (const auto &p : paulis) {
          if (p.size() != sv.n_) throw py::value_error("Pauli string length must equal num_qubits");
          flat += p;
        }
        double out = 0;
        py::gil_scoped_release nogil;
        check(sq_expect_pauli(sv.dev(), flat.data(), weights.data(), uint32_t(weights.size()), &out,
                              stream_ptr(stream)));
        return out;
      },
      py::arg("state_vector"), py::arg("paulis"), py::arg("weights"), py::kw_only(),
      py::arg("stream") = nullptr);
  m_functionals.def(
      "sample",
      [](StateVector &sv, py::array_t<double, py::array::c_style | py::array::forcecast> uniforms,
         std::shared_ptr<Stream> stream) {
        auto u = uniforms.unchecked<1>();
        py::array_t<uint64_t> out(u.shape(0));
        const double *up = uniforms.data();
        uint64_t *op = out.mutable_data();
        const uint64_t shots = uint64_t(u.shape(0));
        {
          py::gil_scoped_release nogil;
          check(sq_sample_host(sv.dev(), up, shots, op, stream_ptr(stream)));
        }
        return out;
      },
      py::arg("state_vector"), py::arg("uniforms"), py::kw_only(), py::arg("stream") = nullptr,
      "Measurement shots on the device: basis-state indices at the given uniforms in [0, 1).");
  m_functionals.def(
      "set_option",
      [](StateVector &sv, int option, int64_t value) { check(sq_set_option(sv.dev(), option, value)); },
      py::arg("state_vector"), py::arg("option"), py::arg("value"));
  m_functionals.def("launch_count", [](StateVector &sv) {
    uint64_t c = 0;
    check(sq_launch_count(sv.dev(), &c));
    return c;
  });

  // StateVector
  auto m_result_types = m.def_submodule("result_types");
  py::class_<StateVector, std::shared_ptr<StateVector>>(m_result_types, "StateVector",
                                                        py::buffer_protocol())
      .def_buffer(&StateVector::buffer)
      .def(py::init<size_t>())
      .def(py::init<size_t, bool>())
      .def(py::init<DeviceType, size_t>())
      .def(py::init([](DeviceType d, size_t n, const std::string &precision) {
             if (precision != "complex128" && precision != "complex64")
               throw py::value_error("precision must be 'complex128' or 'complex64'");
             return std::make_shared<StateVector>(d, n, false,
                                                  precision == "complex64" ? SQ_C64 : SQ_C128);
           }),
           py::arg("device"), py::arg("num_qubits"), py::arg("precision"))
      // A host (optionally pinned) state of either precision, e.g. the
      // destination of a complex64 device state's copy.
      .def(py::init([](size_t n, bool pinned, const std::string &precision) {
             if (precision != "complex128" && precision != "complex64")
               throw py::value_error("precision must be 'complex128' or 'complex64'");
             return std::make_shared<StateVector>(DeviceType::CPU, n, pinned,
                                                  precision == "complex64" ? SQ_C64 : SQ_C128);
           }),
           py::arg("num_qubits"), py::arg("pinned"), py::arg("precision"))
      .def("cpu", &StateVector::cpu, py::kw_only(), py::arg("stream") = nullptr)
      .def("cuda", &StateVector::cuda, py::kw_only(), py::arg("stream") = nullptr)
      .def("copy", &StateVector::copy, py::arg("other"), py::kw_only(), py::arg("stream") = nullptr)
      .def("slice", &StateVector::slice)
      .def("__repr__", &StateVector::formatted_string)
      .def("num_elems", [](const StateVector &s) { return size_t(1) << s.n_; })
      .def("num_qubits", [](const StateVector &s) { return s.n_; })
      .def("sync", &StateVector::sync)
      .def_property_readonly("device", [](const StateVector &s) { return s.dev_; })
      .def_property_readonly("precision", [](const StateVector &s) {
        return std::string(s.dtype_ == SQ_C64 ? "complex64" : "complex128");
      })
      .def("data_ptr", [](const StateVector &s) {
        return reinterpret_cast<uintptr_t>(s.dev_ == DeviceType::CUDA ? sq_state_data(s.ds_->s) : s.host_);
      });

  // Core (core/runtime.cc:33-40, core/cuda/runtime.cu:4-25)
  auto m_core = m.def_submodule("core");
  m_core.def("mem_info", []() {
    const size_t page = size_t(sysconf(_SC_PAGESIZE));
    return std::make_pair(size_t(sysconf(_SC_AVPHYS_PAGES)) * page,
                          size_t(sysconf(_SC_PHYS_PAGES)) * page);
  });
  auto m_core_cuda = m_core.def_submodule("cuda");
  m_core_cuda.def("mem_info", []() {
    size_t f = 0, t = 0;
    check(sq_mem_info(&f, &t));
    return std::make_pair(f, t);
  });
  m_core_cuda.def("device_count", []() {
    int c = 0;
    check(sq_device_count(&c));
    return c;
  });
  m_core_cuda.def("get_device", []() {
    int d = 0;
    check(sq_get_device(&d));
    return d;
  });
  m_core_cuda.def("set_device", [](int d) { check(sq_set_device(d)); });
  m_core_cuda.def("device_synchronize", []() {
    py::gil_scoped_release nogil;
    check(sq_device_synchronize());
  });
  m.def("version", []() { return std::string(sq_version()); });
}
