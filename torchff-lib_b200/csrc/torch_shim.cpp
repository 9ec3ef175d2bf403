// TorchScript binding of the fused system for C++ hosts: the custom class
// torch.classes.torchff_b200.System, loadable with torch.ops.load_library /
// torch::jit::load without Python (OpenMM-Torch's TorchForce runs a saved TorchScript
// module in C++; the reference's route is examples/tip3p/md.py:449-541, which traces
// Tip3pTorchFF built on its C++-registered ops).
//
//   sys = torch.classes.torchff_b200.System(charges, sigma, epsilon, exclusions, cutoff,
//                                           ewald_alpha, pme_grid, mixed, coul_constant)
//   sys.set_bonded(bonds, b0, kb, angles, theta0, ktheta)   # optional, flexible models
//   e = sys.energy(coords, box)              # 0-d, differentiable in coords (forces)
//   e, f = sys.energy_forces(coords, box)    # f = -dE/dx, no autograd
//
// Parameters are CPU or CUDA tensors (copied at construction); the device system is built
// on the device of the first coordinates it sees. The class pickles its construction
// arguments, so a scripted module holding it can be saved and loaded. Every call runs on
// the current CUDA stream of the coordinates' device and calls the C ABI of libtffb200.
#include <torch/custom_class.h>
#include <torch/script.h>

#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>

#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "tffb200.h"

namespace {

void check(int status, const char *what) {
  if (status != TFF_OK) throw std::runtime_error(std::string(what) + ": " + tff_last_error());
}

at::Tensor host64(const at::Tensor &t) { return t.detach().to(at::kCPU, at::kDouble).contiguous(); }
at::Tensor host_i64(const at::Tensor &t) { return t.detach().to(at::kCPU, at::kLong).contiguous(); }

struct System : torch::CustomClassHolder {
  at::Tensor charges, sigma, epsilon, exclusions;
  double cutoff, alpha, kc;
  int64_t grid, mixed;
  at::Tensor bonds, b0, kb, angles, th0, kth;  // empty when the model has no bonded terms
  tff_system h = nullptr;
  int device = -1;
  std::mutex mu;

  System(at::Tensor q, at::Tensor s, at::Tensor e, at::Tensor excl, double rc, double a, int64_t K, int64_t mixed_,
         double k)
      : charges(host64(q)), sigma(host64(s)), epsilon(host64(e)), exclusions(host_i64(excl).reshape({-1, 2})),
        cutoff(rc), alpha(a), kc(k), grid(K), mixed(mixed_) {
    TORCH_CHECK(charges.numel() == sigma.numel() && charges.numel() == epsilon.numel(),
                "charges, sigma and epsilon need one value per atom");
  }
  ~System() override {
    if (h) tff_system_destroy(h);
  }

  void set_bonded(at::Tensor bd, at::Tensor b0_, at::Tensor kb_, at::Tensor an, at::Tensor th0_, at::Tensor kth_) {
    std::lock_guard<std::mutex> lk(mu);
    bonds = host_i64(bd).reshape({-1, 2});
    b0 = host64(b0_);
    kb = host64(kb_);
    angles = host_i64(an).reshape({-1, 3});
    th0 = host64(th0_);
    kth = host64(kth_);
    if (h) upload_bonded();
  }

  void upload_bonded() {
    if (!bonds.defined()) return;
    check(tff_system_set_bonded(h, bonds.size(0), bonds.data_ptr<int64_t>(), b0.data_ptr<double>(),
                                kb.data_ptr<double>(), angles.size(0), angles.data_ptr<int64_t>(),
                                th0.data_ptr<double>(), kth.data_ptr<double>()),
          "tff_system_set_bonded");
  }

  // The device system, created on `dev` at the first call.
  tff_system handle(int dev) {
    std::lock_guard<std::mutex> lk(mu);
    if (h && dev != device) throw std::runtime_error("torchff_b200.System is bound to another CUDA device");
    if (!h) {
      c10::cuda::CUDAGuard g(dev);
      tff_system_desc d{};
      d.dtype = mixed ? TFF_F32 : TFF_F64;
      d.natoms = charges.numel();
      d.cutoff = cutoff;
      d.ewald_alpha = alpha;
      d.pme_grid = (int)grid;
      d.coul_constant = kc;
      d.max_cluster_neighbors = 0;
      check(tff_system_create(&d, charges.data_ptr<double>(), sigma.data_ptr<double>(), epsilon.data_ptr<double>(),
                              exclusions.size(0), exclusions.data_ptr<int64_t>(), &h),
            "tff_system_create");
      device = dev;
      upload_bonded();
    }
    return h;
  }

  // energy (0-d, coords dtype) and forces (N,3, coords dtype)
  std::tuple<at::Tensor, at::Tensor> evaluate(const at::Tensor &coords, const at::Tensor &box) {
    TORCH_CHECK(coords.is_cuda() && box.is_cuda(), "coords and box must be CUDA tensors");
    TORCH_CHECK(coords.dim() == 2 && coords.size(0) == charges.numel() && coords.size(1) == 3,
                "coords must be (natoms, 3)");
    const int dev = coords.get_device();
    tff_system sys = handle(dev);
    c10::cuda::CUDAGuard g(dev);
    const auto st = mixed ? at::kFloat : at::kDouble;
    at::Tensor x = coords.detach().to(st).contiguous();
    at::Tensor b = box.detach().to(coords.device(), st).contiguous();
    at::Tensor energy = at::empty({1}, coords.options().dtype(at::kDouble));
    at::Tensor forces = at::empty_like(x);
    check(tff_system_eval(sys, x.data_ptr(), b.data_ptr(), energy.data_ptr<double>(), forces.data_ptr(), nullptr,
                          nullptr, (tff_stream_t)c10::cuda::getCurrentCUDAStream(dev).stream()),
          "tff_system_eval");
    return {energy.reshape({}).to(coords.scalar_type()), forces.to(coords.scalar_type())};
  }
};

class SystemEnergy : public torch::autograd::Function<SystemEnergy> {
 public:
  static at::Tensor forward(torch::autograd::AutogradContext *ctx, at::Tensor coords, at::Tensor box,
                            c10::intrusive_ptr<System> sys) {
    auto [e, f] = sys->evaluate(coords, box);
    ctx->save_for_backward({f});
    return e;
  }
  static torch::autograd::variable_list backward(torch::autograd::AutogradContext *ctx,
                                                 torch::autograd::variable_list g) {
    const at::Tensor f = ctx->get_saved_variables()[0];
    return {-f * g[0], at::Tensor(), at::Tensor()};
  }
};

using State = std::tuple<at::Tensor, at::Tensor, at::Tensor, at::Tensor, double, double, int64_t, int64_t, double,
                         std::vector<at::Tensor>>;

}  // namespace

TORCH_LIBRARY(torchff_b200, m) {
  m.class_<System>("System")
      .def(torch::init<at::Tensor, at::Tensor, at::Tensor, at::Tensor, double, double, int64_t, int64_t, double>())
      .def("set_bonded", &System::set_bonded)
      .def("energy",
           [](const c10::intrusive_ptr<System> &self, at::Tensor coords, at::Tensor box) {
             return SystemEnergy::apply(coords, box, self);
           })
      .def("energy_forces",
           [](const c10::intrusive_ptr<System> &self, at::Tensor coords, at::Tensor box) {
             return self->evaluate(coords, box);
           })
      .def("natoms", [](const c10::intrusive_ptr<System> &self) { return self->charges.numel(); })
      .def_pickle(
          [](const c10::intrusive_ptr<System> &s) -> State {
            std::vector<at::Tensor> bonded;
            if (s->bonds.defined()) bonded = {s->bonds, s->b0, s->kb, s->angles, s->th0, s->kth};
            return State(s->charges, s->sigma, s->epsilon, s->exclusions, s->cutoff, s->alpha, s->grid, s->mixed,
                         s->kc, bonded);
          },
          [](State st) -> c10::intrusive_ptr<System> {
            auto s = c10::make_intrusive<System>(std::get<0>(st), std::get<1>(st), std::get<2>(st), std::get<3>(st),
                                                 std::get<4>(st), std::get<5>(st), std::get<6>(st), std::get<7>(st),
                                                 std::get<8>(st));
            const auto &bd = std::get<9>(st);
            if (bd.size() == 6) s->set_bonded(bd[0], bd[1], bd[2], bd[3], bd[4], bd[5]);
            return s;
          });
}
