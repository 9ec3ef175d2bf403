// torch.ops.torchff.* registered from C++ on libtffb200: the reference's operator schemas
// (csrc/nblist/nblist_interface.cpp:4-9, csrc/nonbonded/nonbonded_interface.cpp:4-11,
// csrc/coulomb/coulomb_interface.cpp:5-7, csrc/vdw/vdw_interface.cpp:5-8,
// csrc/multipoles/multipoles_interface.cpp:5-9, csrc/pme/pme_interface.cpp:5-14,
// csrc/bond/bond_interface.cpp:5-6, csrc/angle/angle_interface.cpp:5-8) with the same
// dispatch keys: neighbour lists and force accumulators on CUDA, energy terms on
// AutogradCUDA (plus CUDA for calls without autograd).
//
// Registered in C++, the ops run wherever libtorch runs: a TorchScript module traced or
// scripted over them (the reference's route into OpenMM-Torch, examples/tip3p/md.py:449-541)
// loads in a C++ host that loads this library, with no Python. The Python package loads the
// same library, so both reach one implementation.
//
// As in the reference, each energy op computes the energy and every requested first
// derivative in one forward launch, and backward scales the saved derivatives by the
// incoming gradient (csrc/nonbonded/nonbonded_atom_pairs_cuda.cu:220-237). Output shapes
// follow the reference: (1,) for the nonbonded and Coulomb ops, 0-d for LJ, multipolar, PME,
// bonds and angles. Only rank-0 (point charge) multipolar/PME calls and Lennard-Jones vdW
// are implemented; other ranks and the buffered 14-7 potential raise NotImplementedError.
#include <ATen/ATen.h>
#include <torch/autograd.h>
#include <torch/library.h>

#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>

#include <map>
#include <mutex>
#include <optional>
#include <string>
#include <tuple>

#include "tffb200.h"

namespace {

using torch::autograd::AutogradContext;
using torch::autograd::variable_list;
using OptT = std::optional<at::Tensor>;

const char *status_name(int st) {
  switch (st) {
    case TFF_ERR_INVALID: return "invalid argument";
    case TFF_ERR_CUDA: return "CUDA error";
    case TFF_ERR_CUFFT: return "cuFFT error";
    case TFF_ERR_WORKSPACE: return "workspace too small";
    case TFF_ERR_CAPACITY: return "capacity overflow";
    case TFF_ERR_TIMEOUT: return "timeout";
    default: return "error";
  }
}

void check(int st, const char *what) {
  TORCH_CHECK(st == TFF_OK, what, ": ", status_name(st), ": ", tff_last_error());
}

int dtype_code(const at::Tensor &x) {
  if (x.scalar_type() == at::kFloat) return TFF_F32;
  if (x.scalar_type() == at::kDouble) return TFF_F64;
  TORCH_CHECK_TYPE(false, "unsupported dtype ", x.scalar_type(), "; expected float32 (mixed precision) or float64");
  return -1;
}

void require_cuda(std::initializer_list<const at::Tensor *> ts) {
  for (const at::Tensor *t : ts)
    TORCH_CHECK(t == nullptr || !t->defined() || t->is_cuda(), "torchff_b200 operators need CUDA tensors");
}

const at::Tensor *opt_ptr(const OptT &t) { return t.has_value() && t->defined() ? &*t : nullptr; }

// detached contiguous copy in the given type (a view when nothing changes)
at::Tensor cont(const at::Tensor &t, at::ScalarType st) { return t.detach().to(st).contiguous(); }
at::Tensor cont(const at::Tensor &t) { return t.detach().contiguous(); }
at::Tensor as_long(const at::Tensor &t) { return cont(t, at::kLong); }
std::optional<at::Tensor> as_long(const OptT &t) {
  if (!opt_ptr(t)) return std::nullopt;
  return as_long(*t);
}

void *ptr(const at::Tensor &t) { return t.defined() ? t.data_ptr() : nullptr; }
void *ptr(const std::optional<at::Tensor> &t) { return t.has_value() && t->defined() ? t->data_ptr() : nullptr; }
template <class P>
P *typed(const at::Tensor &t) {
  return t.defined() ? static_cast<P *>(t.data_ptr()) : nullptr;
}
template <class P>
P *typed(const std::optional<at::Tensor> &t) {
  return t.has_value() && t->defined() ? static_cast<P *>(t->data_ptr()) : nullptr;
}

tff_stream_t stream_of(const at::Tensor &x) {
  return (tff_stream_t)c10::cuda::getCurrentCUDAStream(x.device().index()).stream();
}

at::Tensor workspace(size_t bytes, const at::Tensor &like) {
  return at::empty({(int64_t)std::max<size_t>(bytes, 256)}, like.options().dtype(at::kByte));
}

at::Tensor empty_if(bool want, const at::Tensor &like) { return want ? at::empty_like(like) : at::Tensor(); }

// Bit k set: differentiable input k of the list needs its gradient, as Python's
// ctx.needs_input_grad reads it (grad mode on and the input requires grad). Taken before
// Function::apply, which runs forward with grad mode off.
int64_t needs(std::initializer_list<const at::Tensor *> ts) {
  int64_t m = 0, k = 0;
  const bool on = at::GradMode::is_enabled();
  for (const at::Tensor *t : ts) {
    if (on && t->defined() && t->requires_grad()) m |= int64_t(1) << k;
    ++k;
  }
  return m;
}
bool bit(int64_t m, int k) { return (m >> k) & 1; }

at::Tensor scaled(const at::Tensor &g, const at::Tensor &go) { return g.defined() ? g.mul(go) : at::Tensor(); }

void rank0_only(const OptT &p, const OptT &t, const char *what) {
  TORCH_CHECK_NOT_IMPLEMENTED(!opt_ptr(p) && !opt_ptr(t), what, ": only rank 0 (point charges) is implemented");
}

// ---------------------------------------------------------------------------------------
// neighbour lists (CUDA, no autograd: csrc/nblist/nblist_nsquared_cuda.cu:201)
// ---------------------------------------------------------------------------------------

at::Tensor nblist_into(bool cell_list, const at::Tensor &coords, const OptT &box, double cutoff,
                       const at::Tensor &pairs, const OptT &rp, const OptT &col, bool include_self) {
  require_cuda({&coords, opt_ptr(box), &pairs, opt_ptr(rp), opt_ptr(col)});
  c10::cuda::CUDAGuard guard(coords.device());
  const at::Tensor x = cont(coords);
  const int dt = dtype_code(x);
  TORCH_CHECK(pairs.scalar_type() == at::kLong && pairs.is_contiguous() && pairs.dim() == 2 && pairs.size(1) == 2,
              "pairs must be a contiguous (max_npairs, 2) int64 tensor");
  const OptT b = opt_ptr(box) ? OptT(cont(*box, x.scalar_type())) : std::nullopt;
  const OptT r = as_long(rp), c = as_long(col);
  const int64_t n = x.size(0);
  at::Tensor npairs = at::zeros({1}, x.options().dtype(at::kInt));
  if (!cell_list) {
    check(tff_nblist_nsquared(dt, n, ptr(x), ptr(b), cutoff, typed<const int64_t>(r), typed<const int64_t>(c),
                              include_self ? 1 : 0, typed<int64_t>(pairs), pairs.size(0), typed<int32_t>(npairs),
                              stream_of(x)),
          "build_neighbor_list_nsquared");
  } else {
    TORCH_CHECK(b.has_value(), "Cell-list neighbor list requires a periodic box");
    at::Tensor ws = workspace(tff_nblist_cell_list_workspace_bytes(dt, n, 0), x);
    check(tff_nblist_cell_list(dt, n, ptr(x), ptr(b), cutoff, typed<const int64_t>(r), typed<const int64_t>(c),
                               include_self ? 1 : 0, typed<int64_t>(pairs), pairs.size(0), typed<int32_t>(npairs), 0,
                               ptr(ws), (size_t)ws.numel(), stream_of(x)),
          "build_neighbor_list_cell_list");
  }
  return npairs;
}

int64_t pair_capacity(int64_t n, const at::Scalar &max_npairs) {
  const int64_t m = max_npairs.toLong();
  return m < 0 ? n * (n + 1) / 2 : m;
}

std::tuple<at::Tensor, at::Tensor> nblist_nsquared(const at::Tensor &coords, const OptT &box, const at::Scalar &cutoff,
                                                   const at::Scalar &max_npairs, const OptT &rp, const OptT &col,
                                                   bool include_self) {
  at::Tensor pairs = at::empty({pair_capacity(coords.size(0), max_npairs), 2}, coords.options().dtype(at::kLong));
  at::Tensor np = nblist_into(false, coords, box, cutoff.toDouble(), pairs, rp, col, include_self);
  return {pairs, np};
}

at::Tensor nblist_nsquared_out(const at::Tensor &coords, const OptT &box, const at::Scalar &cutoff,
                               const at::Tensor &pairs, const OptT &rp, const OptT &col, bool include_self) {
  return nblist_into(false, coords, box, cutoff.toDouble(), pairs, rp, col, include_self);
}

std::tuple<at::Tensor, at::Tensor> nblist_cell(const at::Tensor &coords, const OptT &box, const at::Scalar &cutoff,
                                               const at::Scalar &max_npairs, const OptT &rp, const OptT &col,
                                               bool include_self) {
  at::Tensor pairs = at::empty({pair_capacity(coords.size(0), max_npairs), 2}, coords.options().dtype(at::kLong));
  at::Tensor np = nblist_into(true, coords, box, cutoff.toDouble(), pairs, rp, col, include_self);
  return {pairs, np};
}

std::tuple<at::Tensor, at::Tensor> nblist_cell_out(const at::Tensor &coords, const OptT &box,
                                                   const at::Scalar &cutoff, const at::Tensor &pairs, const OptT &rp,
                                                   const OptT &col, bool include_self) {
  at::Tensor np = nblist_into(true, coords, box, cutoff.toDouble(), pairs, rp, col, include_self);
  return {pairs, np};
}

// ---------------------------------------------------------------------------------------
// pair energy terms
// ---------------------------------------------------------------------------------------

at::Tensor pair_ws(const at::Tensor &x, int64_t ntypes = 0) {
  return workspace(tff_pairs_workspace_bytes(dtype_code(x), x.size(0), ntypes), x);
}

// energy (1,) and the requested dE/dx, dE/dsigma, dE/depsilon, dE/dq
struct NonbondedOut { at::Tensor e, gx, gs, ge, gq; };
NonbondedOut nonbonded_run(const at::Tensor &coords, const at::Tensor &pairs, const at::Tensor &box,
                           const at::Tensor &sigma, const at::Tensor &epsilon, const at::Tensor &charges, double kc,
                           double rc, bool do_shift, bool nx, bool ns, bool ne, bool nq) {
  require_cuda({&coords, &pairs, &box, &sigma, &epsilon, &charges});
  c10::cuda::CUDAGuard guard(coords.device());
  const at::Tensor x = cont(coords);
  const auto st = x.scalar_type();
  const at::Tensor p = as_long(pairs), b = cont(box, st), s = cont(sigma, st), e = cont(epsilon, st),
                   q = cont(charges, st);
  NonbondedOut o{at::empty({1}, x.options()), empty_if(nx, x), empty_if(ns, s), empty_if(ne, e), empty_if(nq, q)};
  at::Tensor ws = pair_ws(x);
  check(tff_nonbonded_atom_pairs(dtype_code(x), x.size(0), ptr(x), p.size(0), typed<const int64_t>(p), ptr(b),
                                 ptr(s), ptr(e), ptr(q), kc, rc, do_shift ? 1 : 0, ptr(o.e), ptr(o.gx), ptr(o.gs),
                                 ptr(o.ge), ptr(o.gq), ptr(ws), (size_t)ws.numel(), stream_of(x)),
        "compute_nonbonded_energy_from_atom_pairs");
  return o;
}

struct NonbondedFn : torch::autograd::Function<NonbondedFn> {
  static at::Tensor forward(AutogradContext *ctx, const at::Tensor &coords, const at::Tensor &pairs,
                            const at::Tensor &box, const at::Tensor &sigma, const at::Tensor &epsilon,
                            const at::Tensor &charges, const at::Scalar &kc, const at::Scalar &rc, bool do_shift,
                            int64_t need) {
    NonbondedOut o = nonbonded_run(coords, pairs, box, sigma, epsilon, charges, kc.toDouble(), rc.toDouble(),
                                   do_shift, bit(need, 0), bit(need, 1), bit(need, 2), bit(need, 3));
    ctx->save_for_backward({o.gx, o.gs, o.ge, o.gq});
    return o.e;
  }
  static variable_list backward(AutogradContext *ctx, variable_list g) {
    const auto s = ctx->get_saved_variables();
    return {scaled(s[0], g[0]), {}, {}, scaled(s[1], g[0]), scaled(s[2], g[0]), scaled(s[3], g[0]), {}, {}, {}, {}};
  }
};

at::Tensor nonbonded_autograd(const at::Tensor &coords, const at::Tensor &pairs, const at::Tensor &box,
                              const at::Tensor &sigma, const at::Tensor &epsilon, const at::Tensor &charges,
                              const at::Scalar &kc, const at::Scalar &rc, bool do_shift) {
  return NonbondedFn::apply(coords, pairs, box, sigma, epsilon, charges, kc, rc, do_shift,
                            needs({&coords, &sigma, &epsilon, &charges}));
}

at::Tensor nonbonded_cuda(const at::Tensor &coords, const at::Tensor &pairs, const at::Tensor &box,
                          const at::Tensor &sigma, const at::Tensor &epsilon, const at::Tensor &charges,
                          const at::Scalar &kc, const at::Scalar &rc, bool do_shift) {
  return nonbonded_run(coords, pairs, box, sigma, epsilon, charges, kc.toDouble(), rc.toDouble(), do_shift, false,
                       false, false, false)
      .e;
}

void check_forces(const at::Tensor &forces, const at::Tensor &x) {
  TORCH_CHECK(forces.scalar_type() == x.scalar_type() && forces.is_contiguous() && forces.sizes() == x.sizes(),
              "forces must be a contiguous tensor shaped and typed like coords");
}

void nonbonded_forces(const at::Tensor &coords, const at::Tensor &pairs, const at::Tensor &box,
                      const at::Tensor &sigma, const at::Tensor &epsilon, const at::Tensor &charges,
                      const at::Scalar &kc, const at::Scalar &rc, const at::Tensor &forces) {
  require_cuda({&coords, &pairs, &box, &sigma, &epsilon, &charges, &forces});
  c10::cuda::CUDAGuard guard(coords.device());
  const at::Tensor x = cont(coords);
  const auto st = x.scalar_type();
  check_forces(forces, x);
  const at::Tensor p = as_long(pairs), b = cont(box, st), s = cont(sigma, st), e = cont(epsilon, st),
                   q = cont(charges, st);
  at::Tensor ws = pair_ws(x);
  check(tff_nonbonded_forces_atom_pairs(dtype_code(x), x.size(0), ptr(x), p.size(0), typed<const int64_t>(p), ptr(b),
                                        ptr(s), ptr(e), ptr(q), kc.toDouble(), rc.toDouble(), ptr(forces), ptr(ws),
                                        (size_t)ws.numel(), stream_of(x)),
        "compute_nonbonded_forces_from_atom_pairs");
}

struct CoulombOut { at::Tensor e, gx, gq; };
CoulombOut coulomb_run(const at::Tensor &coords, const at::Tensor &pairs, const at::Tensor &box,
                       const at::Tensor &charges, double kc, double rc, bool do_shift, bool nx, bool nq) {
  require_cuda({&coords, &pairs, &box, &charges});
  c10::cuda::CUDAGuard guard(coords.device());
  const at::Tensor x = cont(coords);
  const auto st = x.scalar_type();
  const at::Tensor p = as_long(pairs), b = cont(box, st), q = cont(charges, st);
  CoulombOut o{at::empty({1}, x.options()), empty_if(nx, x), empty_if(nq, q)};
  at::Tensor ws = pair_ws(x);
  check(tff_coulomb_atom_pairs(dtype_code(x), x.size(0), ptr(x), p.size(0), typed<const int64_t>(p), ptr(b), ptr(q),
                               kc, rc, do_shift ? 1 : 0, ptr(o.e), ptr(o.gx), ptr(o.gq), ptr(ws), (size_t)ws.numel(),
                               stream_of(x)),
        "compute_coulomb_energy");
  return o;
}

struct CoulombFn : torch::autograd::Function<CoulombFn> {
  static at::Tensor forward(AutogradContext *ctx, const at::Tensor &coords, const at::Tensor &pairs,
                            const at::Tensor &box, const at::Tensor &charges, const at::Scalar &kc,
                            const at::Scalar &rc, bool do_shift, int64_t need) {
    CoulombOut o = coulomb_run(coords, pairs, box, charges, kc.toDouble(), rc.toDouble(), do_shift, bit(need, 0),
                               bit(need, 1));
    ctx->save_for_backward({o.gx, o.gq});
    return o.e;
  }
  static variable_list backward(AutogradContext *ctx, variable_list g) {
    const auto s = ctx->get_saved_variables();
    return {scaled(s[0], g[0]), {}, {}, scaled(s[1], g[0]), {}, {}, {}, {}};
  }
};

at::Tensor coulomb_autograd(const at::Tensor &coords, const at::Tensor &pairs, const at::Tensor &box,
                            const at::Tensor &charges, const at::Scalar &kc, const at::Scalar &rc, bool do_shift) {
  return CoulombFn::apply(coords, pairs, box, charges, kc, rc, do_shift, needs({&coords, &charges}));
}

at::Tensor coulomb_cuda(const at::Tensor &coords, const at::Tensor &pairs, const at::Tensor &box,
                        const at::Tensor &charges, const at::Scalar &kc, const at::Scalar &rc, bool do_shift) {
  return coulomb_run(coords, pairs, box, charges, kc.toDouble(), rc.toDouble(), do_shift, false, false).e;
}

struct LJOut { at::Tensor e, gx, gs, ge; };
LJOut lj_run(const at::Tensor &coords, const at::Tensor &pairs, const at::Tensor &box, const at::Tensor &sigma,
             const at::Tensor &epsilon, double rc, const OptT &atom_types, bool nx, bool ns, bool ne) {
  require_cuda({&coords, &pairs, &box, &sigma, &epsilon, opt_ptr(atom_types)});
  c10::cuda::CUDAGuard guard(coords.device());
  const at::Tensor x = cont(coords);
  const auto st = x.scalar_type();
  const at::Tensor p = as_long(pairs), b = cont(box, st), s = cont(sigma, st), e = cont(epsilon, st);
  const OptT types = as_long(atom_types);
  int64_t ntypes = 0;
  if (types.has_value()) {
    TORCH_CHECK(s.dim() == 2 && s.size(0) == s.size(1) && e.sizes() == s.sizes(),
                "with atom_types, sigma/epsilon must be (ntypes, ntypes) tables");
    ntypes = s.size(0);
  } else {
    TORCH_CHECK(s.size(0) == p.size(0) && e.size(0) == p.size(0),
                "without atom_types, sigma/epsilon must be per pair, shape (P,)");
  }
  LJOut o{at::empty({}, x.options()), empty_if(nx, x), empty_if(ns, s), empty_if(ne, e)};
  at::Tensor ws = pair_ws(x, ntypes);
  check(tff_lennard_jones_atom_pairs(dtype_code(x), x.size(0), ptr(x), p.size(0), typed<const int64_t>(p), ptr(b),
                                     ptr(s), ptr(e), rc, typed<const int64_t>(types), ntypes, ptr(o.e), ptr(o.gx),
                                     ptr(o.gs), ptr(o.ge), ptr(ws), (size_t)ws.numel(), stream_of(x)),
        "compute_lennard_jones_energy");
  return o;
}

struct LJFn : torch::autograd::Function<LJFn> {
  static at::Tensor forward(AutogradContext *ctx, const at::Tensor &coords, const at::Tensor &pairs,
                            const at::Tensor &box, const at::Tensor &sigma, const at::Tensor &epsilon,
                            const at::Scalar &rc, const OptT &atom_types, int64_t need) {
    LJOut o = lj_run(coords, pairs, box, sigma, epsilon, rc.toDouble(), atom_types, bit(need, 0), bit(need, 1),
                     bit(need, 2));
    ctx->save_for_backward({o.gx, o.gs, o.ge});
    return o.e;
  }
  static variable_list backward(AutogradContext *ctx, variable_list g) {
    const auto s = ctx->get_saved_variables();
    return {scaled(s[0], g[0]), {}, {}, scaled(s[1], g[0]), scaled(s[2], g[0]), {}, {}, {}};
  }
};

at::Tensor lj_autograd(const at::Tensor &coords, const at::Tensor &pairs, const at::Tensor &box,
                       const at::Tensor &sigma, const at::Tensor &epsilon, const at::Scalar &rc,
                       const OptT &atom_types) {
  return LJFn::apply(coords, pairs, box, sigma, epsilon, rc, atom_types, needs({&coords, &sigma, &epsilon}));
}

at::Tensor lj_cuda(const at::Tensor &coords, const at::Tensor &pairs, const at::Tensor &box, const at::Tensor &sigma,
                   const at::Tensor &epsilon, const at::Scalar &rc, const OptT &atom_types) {
  return lj_run(coords, pairs, box, sigma, epsilon, rc.toDouble(), atom_types, false, false, false).e;
}

at::Tensor vdw147(const at::Tensor &, const at::Tensor &, const at::Tensor &, const at::Tensor &, const at::Tensor &,
                  const at::Scalar &, const OptT &) {
  TORCH_CHECK_NOT_IMPLEMENTED(false, "the AMOEBA buffered 14-7 potential is outside the fixed-charge path");
  return at::Tensor();
}

struct EwaldOut { at::Tensor e, gx, gq; };
EwaldOut ewald_run(const at::Tensor &coords, const at::Tensor &box, const at::Tensor &pairs, const OptT &pairs_excl,
                   const at::Tensor &q, double rc, double alpha, double prefactor, bool nx, bool nq) {
  require_cuda({&coords, &box, &pairs, opt_ptr(pairs_excl), &q});
  c10::cuda::CUDAGuard guard(coords.device());
  const at::Tensor x = cont(coords);
  const auto st = x.scalar_type();
  const at::Tensor p = as_long(pairs), b = cont(box, st), qq = cont(q, st);
  const OptT pe = as_long(pairs_excl);
  EwaldOut o{at::empty({}, x.options()), empty_if(nx, x), empty_if(nq, qq)};
  at::Tensor ws = pair_ws(x);
  check(tff_ewald_real_atom_pairs(dtype_code(x), x.size(0), ptr(x), ptr(b), p.size(0), typed<const int64_t>(p),
                                  pe.has_value() ? pe->size(0) : 0, typed<const int64_t>(pe), ptr(qq), rc, alpha,
                                  prefactor, ptr(o.e), ptr(o.gx), ptr(o.gq), ptr(ws), (size_t)ws.numel(),
                                  stream_of(x)),
        "compute_multipolar_energy_from_atom_pairs");
  return o;
}

struct EwaldFn : torch::autograd::Function<EwaldFn> {
  static at::Tensor forward(AutogradContext *ctx, const at::Tensor &coords, const at::Tensor &box,
                            const at::Tensor &pairs, const OptT &pairs_excl, const at::Tensor &q, const OptT &p,
                            const OptT &t, const at::Scalar &rc, const at::Scalar &alpha, const at::Scalar &prefactor,
                            int64_t need) {
    rank0_only(p, t, "compute_multipolar_energy_from_atom_pairs");
    EwaldOut o = ewald_run(coords, box, pairs, pairs_excl, q, rc.toDouble(), alpha.toDouble(), prefactor.toDouble(),
                           bit(need, 0), bit(need, 1));
    ctx->save_for_backward({o.gx, o.gq});
    return o.e;
  }
  static variable_list backward(AutogradContext *ctx, variable_list g) {
    const auto s = ctx->get_saved_variables();
    return {scaled(s[0], g[0]), {}, {}, {}, scaled(s[1], g[0]), {}, {}, {}, {}, {}, {}};
  }
};

at::Tensor ewald_autograd(const at::Tensor &coords, const at::Tensor &box, const at::Tensor &pairs,
                          const OptT &pairs_excl, const at::Tensor &q, const OptT &p, const OptT &t,
                          const at::Scalar &rc, const at::Scalar &alpha, const at::Scalar &prefactor) {
  return EwaldFn::apply(coords, box, pairs, pairs_excl, q, p, t, rc, alpha, prefactor, needs({&coords, &q}));
}

at::Tensor ewald_cuda(const at::Tensor &coords, const at::Tensor &box, const at::Tensor &pairs,
                      const OptT &pairs_excl, const at::Tensor &q, const OptT &p, const OptT &t, const at::Scalar &rc,
                      const at::Scalar &alpha, const at::Scalar &prefactor) {
  rank0_only(p, t, "compute_multipolar_energy_from_atom_pairs");
  return ewald_run(coords, box, pairs, pairs_excl, q, rc.toDouble(), alpha.toDouble(), prefactor.toDouble(), false,
                   false)
      .e;
}

// ---------------------------------------------------------------------------------------
// PME: one cuFFT plan per (dtype, K, device), kept for the life of the process
// ---------------------------------------------------------------------------------------

tff_pme_plan pme_plan(int dt, int K, int device) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int>, tff_pme_plan> plans;
  std::lock_guard<std::mutex> lk(mu);
  const auto key = std::make_tuple(dt, K, device);
  auto it = plans.find(key);
  if (it != plans.end()) return it->second;
  tff_pme_plan h = nullptr;
  check(tff_pme_plan_create(dt, K, &h), "tff_pme_plan_create");
  plans.emplace(key, h);
  return h;
}

struct PmeOut { at::Tensor e, gx, phi; };
PmeOut pme_run(const at::Tensor &coords, const at::Tensor &box, const at::Tensor &q, int64_t K, double alpha,
               const at::Tensor &xmod, const at::Tensor &ymod, const at::Tensor &zmod, bool nx, bool nq) {
  require_cuda({&coords, &box, &q, &xmod, &ymod, &zmod});
  c10::cuda::CUDAGuard guard(coords.device());
  const at::Tensor x = cont(coords);
  const auto st = x.scalar_type();
  const at::Tensor b = cont(box, st), qq = cont(q, st), xm = cont(xmod, st), ym = cont(ymod, st), zm = cont(zmod, st);
  TORCH_CHECK(xm.numel() == K && ym.numel() == K && zm.numel() == K / 2 + 1,
              "B-spline moduli must have K, K and K//2+1 entries");
  const int dt = dtype_code(x);
  tff_pme_plan plan = pme_plan(dt, (int)K, x.device().index());
  PmeOut o{at::empty({}, x.options()), empty_if(nx, x), empty_if(nq, qq)};
  at::Tensor ws = workspace(tff_pme_workspace_bytes(plan, x.size(0)), x);
  check(tff_pme_long_range(plan, x.size(0), ptr(x), ptr(b), ptr(qq), alpha, ptr(xm), ptr(ym), ptr(zm), ptr(o.e),
                           ptr(o.phi), ptr(o.gx), ptr(ws), (size_t)ws.numel(), stream_of(x)),
        "pme_long_range");
  return o;
}

struct PmeFn : torch::autograd::Function<PmeFn> {
  static at::Tensor forward(AutogradContext *ctx, const at::Tensor &coords, const at::Tensor &box,
                            const at::Tensor &q, const OptT &p, const OptT &t, const at::Scalar &K,
                            const at::Scalar &alpha, const at::Tensor &xmod, const at::Tensor &ymod,
                            const at::Tensor &zmod, int64_t need) {
    rank0_only(p, t, "pme_long_range");
    PmeOut o = pme_run(coords, box, q, K.toLong(), alpha.toDouble(), xmod, ymod, zmod, bit(need, 0), bit(need, 1));
    ctx->save_for_backward({o.gx, o.phi});
    return o.e;
  }
  static variable_list backward(AutogradContext *ctx, variable_list g) {
    const auto s = ctx->get_saved_variables();
    return {scaled(s[0], g[0]), {}, scaled(s[1], g[0]), {}, {}, {}, {}, {}, {}, {}, {}};
  }
};

at::Tensor pme_autograd(const at::Tensor &coords, const at::Tensor &box, const at::Tensor &q, const OptT &p,
                        const OptT &t, const at::Scalar &K, const at::Scalar &alpha, const at::Tensor &xmod,
                        const at::Tensor &ymod, const at::Tensor &zmod) {
  return PmeFn::apply(coords, box, q, p, t, K, alpha, xmod, ymod, zmod, needs({&coords, &q}));
}

at::Tensor pme_cuda(const at::Tensor &coords, const at::Tensor &box, const at::Tensor &q, const OptT &p,
                    const OptT &t, const at::Scalar &K, const at::Scalar &alpha, const at::Tensor &xmod,
                    const at::Tensor &ymod, const at::Tensor &zmod) {
  rank0_only(p, t, "pme_long_range");
  return pme_run(coords, box, q, K.toLong(), alpha.toDouble(), xmod, ymod, zmod, false, false).e;
}

// ---------------------------------------------------------------------------------------
// bonded terms
// ---------------------------------------------------------------------------------------

at::Tensor bonded_ws(const at::Tensor &x, int64_t nterms) {
  return workspace(tff_bonded_workspace_bytes(dtype_code(x), x.size(0), nterms), x);
}

at::Tensor bonded_index(const at::Tensor &idx, bool angle) {
  const at::Tensor ix = as_long(idx);
  TORCH_CHECK(ix.dim() == 2 && ix.size(1) == (angle ? 3 : 2), angle ? "angles" : "bonds", " must be an (M, ",
              angle ? 3 : 2, ") index tensor");
  return ix;
}

struct BondedOut { at::Tensor e, gx, gp, gk; };
BondedOut bonded_run(bool angle, const at::Tensor &coords, const at::Tensor &idx, const at::Tensor &p0,
                     const at::Tensor &k, bool nx, bool np, bool nk) {
  require_cuda({&coords, &idx, &p0, &k});
  c10::cuda::CUDAGuard guard(coords.device());
  const at::Tensor x = cont(coords);
  const auto st = x.scalar_type();
  const at::Tensor ix = bonded_index(idx, angle), a = cont(p0, st), kk = cont(k, st);
  BondedOut o{at::empty({}, x.options()), empty_if(nx, x), empty_if(np, a), empty_if(nk, kk)};
  at::Tensor ws = bonded_ws(x, ix.size(0));
  auto fn = angle ? tff_harmonic_angle : tff_harmonic_bond;
  check(fn(dtype_code(x), x.size(0), ptr(x), ix.size(0), typed<const int64_t>(ix), ptr(a), ptr(kk), ptr(o.e),
           ptr(o.gx), ptr(o.gp), ptr(o.gk), ptr(ws), (size_t)ws.numel(), stream_of(x)),
        angle ? "compute_harmonic_angle_energy" : "compute_harmonic_bond_energy");
  return o;
}

template <bool ANGLE>
struct BondedFn : torch::autograd::Function<BondedFn<ANGLE>> {
  static at::Tensor forward(AutogradContext *ctx, const at::Tensor &coords, const at::Tensor &idx,
                            const at::Tensor &p0, const at::Tensor &k, int64_t need) {
    BondedOut o = bonded_run(ANGLE, coords, idx, p0, k, bit(need, 0), bit(need, 1), bit(need, 2));
    ctx->save_for_backward({o.gx, o.gp, o.gk});
    return o.e;
  }
  static variable_list backward(AutogradContext *ctx, variable_list g) {
    const auto s = ctx->get_saved_variables();
    return {scaled(s[0], g[0]), {}, scaled(s[1], g[0]), scaled(s[2], g[0]), {}};
  }
};

template <bool ANGLE>
at::Tensor bonded_autograd(const at::Tensor &coords, const at::Tensor &idx, const at::Tensor &p0,
                           const at::Tensor &k) {
  return BondedFn<ANGLE>::apply(coords, idx, p0, k, needs({&coords, &p0, &k}));
}

template <bool ANGLE>
at::Tensor bonded_cuda(const at::Tensor &coords, const at::Tensor &idx, const at::Tensor &p0, const at::Tensor &k) {
  return bonded_run(ANGLE, coords, idx, p0, k, false, false, false).e;
}

template <bool ANGLE>
void bonded_forces(const at::Tensor &coords, const at::Tensor &idx, const at::Tensor &p0, const at::Tensor &k,
                   const at::Tensor &forces) {
  require_cuda({&coords, &idx, &p0, &k, &forces});
  c10::cuda::CUDAGuard guard(coords.device());
  const at::Tensor x = cont(coords);
  const auto st = x.scalar_type();
  check_forces(forces, x);
  const at::Tensor ix = as_long(idx), a = cont(p0, st), kk = cont(k, st);
  at::Tensor ws = bonded_ws(x, ix.size(0));
  auto fn = ANGLE ? tff_harmonic_angle_forces : tff_harmonic_bond_forces;
  check(fn(dtype_code(x), x.size(0), ptr(x), ix.size(0), typed<const int64_t>(ix), ptr(a), ptr(kk), ptr(forces),
           ptr(ws), (size_t)ws.numel(), stream_of(x)),
        ANGLE ? "compute_harmonic_angle_forces" : "compute_harmonic_bond_forces");
}

// theta (M,), or with grad_theta the coordinate gradient sum grad_theta dtheta/dx
at::Tensor angles_run(const at::Tensor &coords, const at::Tensor &angles, const at::Tensor &grad_theta) {
  require_cuda({&coords, &angles});
  c10::cuda::CUDAGuard guard(coords.device());
  const at::Tensor x = cont(coords);
  const at::Tensor ix = bonded_index(angles, true);
  const int dt = dtype_code(x);
  if (!grad_theta.defined()) {
    at::Tensor theta = at::empty({ix.size(0)}, x.options());
    check(tff_angles(dt, x.size(0), ptr(x), ix.size(0), typed<const int64_t>(ix), ptr(theta), nullptr, nullptr,
                     nullptr, 0, stream_of(x)),
          "compute_angles");
    return theta;
  }
  const at::Tensor gt = cont(grad_theta, x.scalar_type());
  at::Tensor gx = at::empty_like(x);
  at::Tensor ws = bonded_ws(x, ix.size(0));
  check(tff_angles(dt, x.size(0), ptr(x), ix.size(0), typed<const int64_t>(ix), nullptr, ptr(gt), ptr(gx), ptr(ws),
                   (size_t)ws.numel(), stream_of(x)),
        "compute_angles backward");
  return gx;
}

struct AnglesFn : torch::autograd::Function<AnglesFn> {
  static at::Tensor forward(AutogradContext *ctx, const at::Tensor &coords, const at::Tensor &angles) {
    ctx->save_for_backward({coords, angles});
    return angles_run(coords, angles, at::Tensor());
  }
  static variable_list backward(AutogradContext *ctx, variable_list g) {
    const auto s = ctx->get_saved_variables();
    return {angles_run(s[0], s[1], g[0]), {}};
  }
};

at::Tensor angles_autograd(const at::Tensor &coords, const at::Tensor &angles) {
  return AnglesFn::apply(coords, angles);
}
at::Tensor angles_cuda(const at::Tensor &coords, const at::Tensor &angles) {
  return angles_run(coords, angles, at::Tensor());
}

}  // namespace

TORCH_LIBRARY_FRAGMENT(torchff, m) {
  m.def("build_neighbor_list_nsquared(Tensor coords, Tensor? box, Scalar cutoff, Scalar max_npairs, "
        "Tensor? excl_row_ptr, Tensor? excl_col_indices, bool include_self) -> (Tensor, Tensor)");
  m.def("build_neighbor_list_nsquared_out(Tensor coords, Tensor? box, Scalar cutoff, Tensor(a!) pairs, "
        "Tensor? excl_row_ptr, Tensor? excl_col_indices, bool include_self) -> Tensor");
  m.def("build_neighbor_list_cell_list(Tensor coords, Tensor? box, Scalar cutoff, Scalar max_npairs, "
        "Tensor? excl_row_ptr, Tensor? excl_col_indices, bool include_self) -> (Tensor, Tensor)");
  m.def("build_neighbor_list_cell_list_out(Tensor coords, Tensor? box, Scalar cutoff, Tensor(a!) pairs, "
        "Tensor? excl_row_ptr, Tensor? excl_col_indices, bool include_self) -> (Tensor, Tensor)");
  m.def("compute_nonbonded_energy_from_atom_pairs(Tensor coords, Tensor pairs, Tensor box, Tensor sigma, "
        "Tensor epsilon, Tensor charges, Scalar coul_constant, Scalar cutoff, bool do_shift) -> Tensor");
  m.def("compute_nonbonded_forces_from_atom_pairs(Tensor coords, Tensor pairs, Tensor box, Tensor sigma, "
        "Tensor epsilon, Tensor charges, Scalar coul_constant, Scalar cutoff, Tensor forces) -> ()");
  m.def("compute_coulomb_energy(Tensor coords, Tensor pairs, Tensor box, Tensor charges, Scalar coulomb_constant, "
        "Scalar cutoff, bool do_shift) -> Tensor");
  m.def("compute_lennard_jones_energy(Tensor coords, Tensor pairs, Tensor box, Tensor sigma, Tensor epsilon, "
        "Scalar cutoff, Tensor? atom_types) -> Tensor");
  m.def("compute_vdw_14_7_energy(Tensor coords, Tensor pairs, Tensor box, Tensor radius, Tensor epsilon, "
        "Scalar cutoff, Tensor? atom_types) -> Tensor");
  m.def("compute_multipolar_energy_from_atom_pairs(Tensor coords, Tensor box, Tensor pairs, Tensor? pairs_excl, "
        "Tensor q, Tensor? p, Tensor? t, Scalar cutoff, Scalar ewald_alpha, Scalar prefactor) -> Tensor");
  m.def("compute_harmonic_bond_energy(Tensor coords, Tensor pairs, Tensor b0, Tensor k) -> Tensor");
  m.def("compute_harmonic_bond_forces(Tensor coords, Tensor pairs, Tensor b0, Tensor k, Tensor(a!) forces) -> ()");
  m.def("compute_harmonic_angle_energy(Tensor coords, Tensor angles, Tensor theta0, Tensor k) -> Tensor");
  m.def("compute_harmonic_angle_forces(Tensor coords, Tensor angles, Tensor theta0, Tensor k, "
        "Tensor(a!) forces) -> ()");
  m.def("compute_angles(Tensor coords, Tensor angles) -> Tensor");
  m.def("pme_long_range(Tensor coords, Tensor box, Tensor q, Tensor? p, Tensor? t, Scalar K, Scalar alpha, "
        "Tensor xmoduli, Tensor ymoduli, Tensor zmoduli) -> Tensor");
}

TORCH_LIBRARY_IMPL(torchff, CUDA, m) {
  m.impl("build_neighbor_list_nsquared", nblist_nsquared);
  m.impl("build_neighbor_list_nsquared_out", nblist_nsquared_out);
  m.impl("build_neighbor_list_cell_list", nblist_cell);
  m.impl("build_neighbor_list_cell_list_out", nblist_cell_out);
  m.impl("compute_nonbonded_energy_from_atom_pairs", nonbonded_cuda);
  m.impl("compute_nonbonded_forces_from_atom_pairs", nonbonded_forces);
  m.impl("compute_coulomb_energy", coulomb_cuda);
  m.impl("compute_lennard_jones_energy", lj_cuda);
  m.impl("compute_vdw_14_7_energy", vdw147);
  m.impl("compute_multipolar_energy_from_atom_pairs", ewald_cuda);
  m.impl("compute_harmonic_bond_energy", bonded_cuda<false>);
  m.impl("compute_harmonic_bond_forces", bonded_forces<false>);
  m.impl("compute_harmonic_angle_energy", bonded_cuda<true>);
  m.impl("compute_harmonic_angle_forces", bonded_forces<true>);
  m.impl("compute_angles", angles_cuda);
  m.impl("pme_long_range", pme_cuda);
}

TORCH_LIBRARY_IMPL(torchff, AutogradCUDA, m) {
  m.impl("compute_nonbonded_energy_from_atom_pairs", nonbonded_autograd);
  m.impl("compute_coulomb_energy", coulomb_autograd);
  m.impl("compute_lennard_jones_energy", lj_autograd);
  m.impl("compute_vdw_14_7_energy", vdw147);
  m.impl("compute_multipolar_energy_from_atom_pairs", ewald_autograd);
  m.impl("compute_harmonic_bond_energy", bonded_autograd<false>);
  m.impl("compute_harmonic_angle_energy", bonded_autograd<true>);
  m.impl("compute_angles", angles_autograd);
  m.impl("pme_long_range", pme_autograd);
}
