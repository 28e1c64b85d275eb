// Torch extension `cuda_knn_aggregate._C`: validates tensors, allocates
// outputs and scratch from torch's caching allocator, and calls the C ABI of
// libknn_aniso.so on the current CUDA stream.
//
// The first three ops keep the names, argument lists and return lists of
// the reference's pybind module (csrc/knn_aggregate.cpp:26-47, 101-172,
// 178-185) so code written against it runs unchanged; the *_ex ops expose
// the reuse of packed points, adjacency and coefficients that the autograd
// layer uses.
#include <ATen/cuda/CUDAContext.h>
#include <ATen/cuda/CUDAEvent.h>
#include <c10/cuda/CUDAGuard.h>
#include <torch/extension.h>

#include <cstdlib>
#include <string>
#include <vector>

#include "knn_aniso.h"

namespace {

#define KNN_CHECK_CUDA(x) TORCH_CHECK((x).is_cuda(), #x " must be a CUDA tensor")
#define KNN_CHECK_CONTIGUOUS(x) TORCH_CHECK((x).is_contiguous(), #x " must be contiguous")
#define KNN_CHECK_INPUT(x) \
  KNN_CHECK_CUDA(x);       \
  KNN_CHECK_CONTIGUOUS(x)

void check_status(int rc, const char* what) {
  TORCH_CHECK(rc == KNNAG_OK, what, " failed: ", knnag_status_string(rc));
}

// Opt-in check of the errors the kernels latch on the device (a bounded
// wait that gave up, an internal index out of range): with the environment
// variable KNNAG_CHECK_DEVICE_STATUS set to a value other than "0", every op
// reads its workspace's status word after its launches (which synchronises
// the stream, so such a process cannot capture the ops into a CUDA graph)
// and raises if an error was latched.  Off by default: the ops then neither
// synchronise nor report device-latched errors.
bool device_status_checks() {
  const char* e = std::getenv("KNNAG_CHECK_DEVICE_STATUS");
  return e && e[0] && !(e[0] == '0' && e[1] == 0);
}

void check_device_status(const torch::Tensor& ws, void* stream, const char* what) {
  if (!device_status_checks()) return;
  TORCH_CHECK(knnag_read_device_status(ws.data_ptr(), stream) == KNNAG_OK, what,
              ": an error was latched on the device (", knnag_status_string(KNNAG_ERR_DEVICE), ")");
}

int dtype_code(const torch::Tensor& t) {
  if (t.scalar_type() == torch::kFloat32) return KNNAG_F32;
  if (t.scalar_type() == torch::kFloat64) return KNNAG_F64;
  TORCH_CHECK(false, "knn_aggregate_aniso supports float32 and float64, got ", t.scalar_type());
  return -1;
}

struct Dims {
  int B, Q, P, F, dtype;
};

Dims check_inputs(const torch::Tensor& q, const torch::Tensor& p, const torch::Tensor& f,
                  const torch::Tensor& sigma, const torch::Tensor& R) {
  KNN_CHECK_INPUT(q);
  KNN_CHECK_INPUT(p);
  KNN_CHECK_INPUT(f);
  KNN_CHECK_INPUT(sigma);
  KNN_CHECK_INPUT(R);
  TORCH_CHECK(q.dim() == 3 && q.size(2) == 3, "q must have shape [B, Q, 3]");
  TORCH_CHECK(p.dim() == 3 && p.size(2) == 3, "p must have shape [B, P, 3]");
  const int64_t B = q.size(0), P = p.size(1);
  TORCH_CHECK(p.size(0) == B, "p batch size must match q");
  TORCH_CHECK(f.dim() == 3 && f.size(0) == B && f.size(1) == P, "f must have shape [B, P, F]");
  TORCH_CHECK(sigma.dim() == 3 && sigma.size(0) == B && sigma.size(1) == P && sigma.size(2) == 3,
              "sigma must have shape [B, P, 3]");
  TORCH_CHECK(R.dim() == 4 && R.size(0) == B && R.size(1) == P && R.size(2) == 3 && R.size(3) == 3,
              "R must have shape [B, P, 3, 3]");
  const int dt = dtype_code(q);
  for (const torch::Tensor* t : {&p, &f, &sigma, &R})
    TORCH_CHECK(t->scalar_type() == q.scalar_type(), "all floating-point inputs must share q's dtype");
  for (const torch::Tensor* t : {&p, &f, &sigma, &R})
    TORCH_CHECK(t->device() == q.device(), "all inputs must be on the same device");
  TORCH_CHECK(B <= INT32_MAX && q.size(1) <= INT32_MAX && P <= INT32_MAX && f.size(2) <= INT32_MAX,
              "sizes exceed the 32-bit range");
  return Dims{(int)B, (int)q.size(1), (int)P, (int)f.size(2), dt};
}

void check_k(int64_t K, int P) {
  TORCH_CHECK(K >= 1 && K <= P, "K must satisfy 1 <= K <= P (K=", K, ", P=", P, ")");
}

torch::Tensor scratch(size_t bytes, const torch::Tensor& like) {
  return torch::empty({(int64_t)(bytes > 0 ? bytes : 1)}, like.options().dtype(torch::kUInt8));
}

void* stream_of(const torch::Tensor& t) { return (void*)at::cuda::getCurrentCUDAStream(t.device().index()).stream(); }

void* ptr_or_null(const c10::optional<torch::Tensor>& t) { return (t && t->defined()) ? t->data_ptr() : nullptr; }

// want_adj: also count the point -> entry adjacency's rows in the forward
// (knnag_forward_counted); the buffer is returned last.
std::vector<torch::Tensor> forward_impl(const torch::Tensor& q, const torch::Tensor& p, const torch::Tensor& f,
                                        const torch::Tensor& sigma, const torch::Tensor& R, int64_t K,
                                        bool want_points, bool want_adj = false) {
  const Dims d = check_inputs(q, p, f, sigma, R);
  check_k(K, d.P);
  const c10::cuda::CUDAGuard guard(q.device());
  auto f_out = torch::empty({d.B, d.Q, d.F}, f.options());
  auto w_out = torch::empty({d.B, d.Q, K}, f.options());
  auto dists = torch::empty({d.B, d.Q, K}, q.options());
  auto idxs = torch::empty({d.B, d.Q, K}, q.options().dtype(torch::kInt64));
  torch::Tensor points;
  if (want_points) points = torch::empty({d.B, d.P, 16}, p.options());
  const size_t ws_bytes = knnag_forward_workspace_bytes(d.B, d.Q, d.P, d.F, (int)K, d.dtype);
  auto ws = scratch(ws_bytes, q);
  torch::Tensor adj;
  int rc;
  if (want_adj) {
    adj = scratch(knnag_adjacency_bytes(d.B, d.Q, d.P, (int)K), q);
    rc = knnag_forward_counted(q.data_ptr(), p.data_ptr(), f.data_ptr(), sigma.data_ptr(), R.data_ptr(), d.B, d.Q,
                               d.P, d.F, (int)K, d.dtype, f_out.data_ptr(), w_out.data_ptr(), dists.data_ptr(),
                               idxs.data_ptr<int64_t>(), want_points ? points.data_ptr() : nullptr, adj.data_ptr(),
                               ws.data_ptr(), ws_bytes, stream_of(q));
  } else {
    rc = knnag_forward(q.data_ptr(), p.data_ptr(), f.data_ptr(), sigma.data_ptr(), R.data_ptr(), d.B, d.Q, d.P, d.F,
                       (int)K, d.dtype, f_out.data_ptr(), w_out.data_ptr(), dists.data_ptr(), idxs.data_ptr<int64_t>(),
                       want_points ? points.data_ptr() : nullptr, ws.data_ptr(), ws_bytes, stream_of(q));
  }
  check_status(rc, "knn_aggregate_aniso_forward");
  check_device_status(ws, stream_of(q), "knn_aggregate_aniso_forward");
  std::vector<torch::Tensor> out{f_out, w_out, dists, idxs};
  if (want_points) out.push_back(points);
  if (want_adj) out.push_back(adj);
  return out;
}

void check_idxs(const torch::Tensor& idxs, const Dims& d) {
  KNN_CHECK_INPUT(idxs);
  TORCH_CHECK(idxs.scalar_type() == torch::kInt64, "idxs must be int64");
  TORCH_CHECK(idxs.dim() == 3 && idxs.size(0) == d.B && idxs.size(1) == d.Q, "idxs must have shape [B, Q, K]");
  check_k(idxs.size(2), d.P);
}

void check_like(const torch::Tensor& t, const char* name, std::vector<int64_t> shape, const torch::Tensor& ref) {
  TORCH_CHECK(t.is_cuda(), name, " must be a CUDA tensor");
  TORCH_CHECK(t.is_contiguous(), name, " must be contiguous");
  TORCH_CHECK(t.sizes() == c10::IntArrayRef(shape), name, " has the wrong shape");
  TORCH_CHECK(t.scalar_type() == ref.scalar_type(), name, " must share q's dtype");
}

// needs bits -> output tensors (undefined tensors for skipped outputs)
std::vector<torch::Tensor> backward_impl(int order, const c10::optional<torch::Tensor>& ggq, const torch::Tensor& gfo,
                                         const torch::Tensor& q, const torch::Tensor& p, const torch::Tensor& f,
                                         const torch::Tensor& sigma, const torch::Tensor& R,
                                         const c10::optional<torch::Tensor>& w_out, const torch::Tensor& idxs,
                                         const c10::optional<torch::Tensor>& points,
                                         const c10::optional<torch::Tensor>& adjacency,
                                         const c10::optional<torch::Tensor>& coef, int64_t needs, bool want_coef) {
  const Dims d = check_inputs(q, p, f, sigma, R);
  check_idxs(idxs, d);
  const int K = (int)idxs.size(2);
  if (needs & KNNAG_GFO_SCALAR) {
    // one value broadcast over [B, Q, F]: the kernels read gfo.data_ptr()[0]
    TORCH_CHECK(gfo.is_cuda() && gfo.numel() > 0 && gfo.scalar_type() == q.scalar_type(),
                "broadcast grad_f_out must be a CUDA tensor of q's dtype");
  } else {
    check_like(gfo, "grad_f_out", {d.B, d.Q, d.F}, q);
  }
  if (order == 2) check_like(*ggq, "grad_grad_q", {d.B, d.Q, 3}, q);
  if (w_out && w_out->defined()) check_like(*w_out, "w_out", {d.B, d.Q, K}, q);
  if (points && points->defined()) check_like(*points, "points", {d.B, d.P, 16}, q);
  if (coef && coef->defined()) check_like(*coef, "coef", {d.B, d.Q, K}, q);
  if (adjacency && adjacency->defined()) {
    TORCH_CHECK(adjacency->is_cuda() && adjacency->scalar_type() == torch::kUInt8 &&
                    (size_t)adjacency->numel() >= knnag_adjacency_bytes(d.B, d.Q, d.P, K),
                "adjacency must be the uint8 CUDA buffer built by build_adjacency");
  }
  const c10::cuda::CUDAGuard guard(q.device());
  torch::Tensor dgfo, dq, dp, df, ds, dR, cf;
  if (order == 2 && (needs & KNNAG_NEED_DGFO)) dgfo = torch::empty({d.B, d.Q, d.F}, f.options());
  if (needs & KNNAG_NEED_DQ) dq = torch::empty({d.B, d.Q, 3}, q.options());
  if (needs & KNNAG_NEED_DP) dp = torch::empty({d.B, d.P, 3}, p.options());
  if (needs & KNNAG_NEED_DF) df = torch::empty({d.B, d.P, d.F}, f.options());
  if (needs & KNNAG_NEED_DSIGMA) ds = torch::empty({d.B, d.P, 3}, sigma.options());
  if (needs & KNNAG_NEED_DR) dR = torch::empty({d.B, d.P, 3, 3}, R.options());
  if (order == 1 && want_coef) cf = torch::empty({d.B, d.Q, K}, q.options());
  auto P_ = [](const torch::Tensor& t) -> void* { return t.defined() ? t.data_ptr() : nullptr; };
  const size_t ws_bytes = knnag_backward_workspace_bytes(d.B, d.Q, d.P, d.F, K, d.dtype);
  auto ws = scratch(ws_bytes, q);
  int rc;
  if (order == 1) {
    rc = knnag_backward(gfo.data_ptr(), nullptr, q.data_ptr(), p.data_ptr(), f.data_ptr(), sigma.data_ptr(),
                        R.data_ptr(), ptr_or_null(w_out), idxs.data_ptr<int64_t>(), d.B, d.Q, d.P, d.F, K, d.dtype,
                        (int)needs, ptr_or_null(points), ptr_or_null(adjacency), P_(dq), P_(dp), P_(df), P_(ds),
                        P_(dR), P_(cf), ws.data_ptr(), ws_bytes, stream_of(q));
    check_status(rc, "knn_aggregate_aniso_backward");
    check_device_status(ws, stream_of(q), "knn_aggregate_aniso_backward");
    return {dq, dp, df, ds, dR, cf};
  }
  rc = knnag_backward_2nd(ggq->data_ptr(), gfo.data_ptr(), nullptr, q.data_ptr(), p.data_ptr(), f.data_ptr(),
                          sigma.data_ptr(), R.data_ptr(), ptr_or_null(w_out), idxs.data_ptr<int64_t>(), d.B, d.Q,
                          d.P, d.F, K, d.dtype, (int)needs, ptr_or_null(points), ptr_or_null(adjacency),
                          ptr_or_null(coef), P_(dgfo), P_(dq), P_(dp), P_(df), P_(ds), P_(dR), ws.data_ptr(),
                          ws_bytes, stream_of(q));
  check_status(rc, "knn_aggregate_aniso_backward_2nd");
  check_device_status(ws, stream_of(q), "knn_aggregate_aniso_backward_2nd");
  return {dgfo, dq, dp, df, ds, dR};
}

// ----------------------------------------------- reference-compatible ops

std::vector<torch::Tensor> knn_aggregate_aniso_forward(torch::Tensor q, torch::Tensor p, torch::Tensor f,
                                                       torch::Tensor sigma, torch::Tensor R, int64_t K) {
  return forward_impl(q, p, f, sigma, R, K, false);
}

std::vector<torch::Tensor> knn_aggregate_aniso_backward(torch::Tensor grad_f_out, torch::Tensor grad_w_out,
                                                        torch::Tensor q, torch::Tensor p, torch::Tensor f,
                                                        torch::Tensor sigma, torch::Tensor R, torch::Tensor w_out,
                                                        torch::Tensor k_idxs) {
  KNN_CHECK_INPUT(grad_f_out);
  KNN_CHECK_INPUT(grad_w_out);
  KNN_CHECK_INPUT(w_out);
  auto r = backward_impl(1, c10::nullopt, grad_f_out, q, p, f, sigma, R, w_out, k_idxs, c10::nullopt, c10::nullopt,
                         c10::nullopt, KNNAG_NEED_DQ | KNNAG_NEED_DP | KNNAG_NEED_DF | KNNAG_NEED_DSIGMA |
                                           KNNAG_NEED_DR,
                         false);
  return {r[0], r[1], r[2], r[3], r[4]};
}

std::vector<torch::Tensor> knn_aggregate_aniso_backward_2nd(torch::Tensor grad_grad_q, torch::Tensor grad_f_out,
                                                            torch::Tensor grad_w_out, torch::Tensor q, torch::Tensor p,
                                                            torch::Tensor f, torch::Tensor sigma, torch::Tensor R,
                                                            torch::Tensor w_out, torch::Tensor k_idxs) {
  KNN_CHECK_INPUT(grad_grad_q);
  KNN_CHECK_INPUT(grad_f_out);
  KNN_CHECK_INPUT(grad_w_out);
  KNN_CHECK_INPUT(w_out);
  return backward_impl(2, grad_grad_q, grad_f_out, q, p, f, sigma, R, w_out, k_idxs, c10::nullopt, c10::nullopt,
                       c10::nullopt, KNNAG_NEED_ALL, false);
}

// ------------------------------------------------- other reference ops

std::vector<torch::Tensor> knn_precomputed_aggregate_aniso_forward(torch::Tensor q, torch::Tensor p, torch::Tensor f,
                                                                   torch::Tensor sigma, torch::Tensor R,
                                                                   torch::Tensor knn_idxs, int64_t K) {
  const Dims d = check_inputs(q, p, f, sigma, R);
  KNN_CHECK_INPUT(knn_idxs);
  TORCH_CHECK(knn_idxs.scalar_type() == torch::kInt64 && knn_idxs.dim() == 3 && knn_idxs.size(0) == d.B &&
                  knn_idxs.size(1) == d.Q && knn_idxs.size(2) == K,
              "knn_idxs must be int64 [B, Q, K]");
  check_k(K, d.P);
  const c10::cuda::CUDAGuard guard(q.device());
  auto f_out = torch::empty({d.B, d.Q, d.F}, f.options());
  auto w_out = torch::empty({d.B, d.Q, K}, f.options());
  auto dists = torch::empty({d.B, d.Q, K}, q.options());
  const size_t nb = knnag_variant_workspace_bytes(d.B, d.Q, d.P, d.dtype);
  auto ws = scratch(nb, q);
  check_status(knnag_forward_precomputed(q.data_ptr(), p.data_ptr(), f.data_ptr(), sigma.data_ptr(), R.data_ptr(),
                                         knn_idxs.data_ptr<int64_t>(), d.B, d.Q, d.P, d.F, (int)K, d.dtype,
                                         f_out.data_ptr(), w_out.data_ptr(), dists.data_ptr(), ws.data_ptr(), nb,
                                         stream_of(q)),
               "knn_precomputed_aggregate_aniso_forward");
  return {f_out, w_out, dists};
}

std::vector<torch::Tensor> knn_lookup_aggregate_aniso_forward(torch::Tensor q, torch::Tensor p, torch::Tensor f,
                                                              torch::Tensor sigma, torch::Tensor R,
                                                              torch::Tensor knn_table, int64_t K) {
  const Dims d = check_inputs(q, p, f, sigma, R);
  KNN_CHECK_INPUT(knn_table);
  TORCH_CHECK(knn_table.scalar_type() == torch::kInt64 && knn_table.dim() == 2 && knn_table.size(0) >= d.P &&
                  knn_table.size(1) >= K,
              "knn_table must be int64 [P, >= K]");
  check_k(K, d.P);
  const c10::cuda::CUDAGuard guard(q.device());
  auto f_out = torch::empty({d.B, d.Q, d.F}, f.options());
  auto w_out = torch::empty({d.B, d.Q, K}, f.options());
  auto dists = torch::empty({d.B, d.Q, K}, q.options());
  auto idxs = torch::empty({d.B, d.Q, K}, q.options().dtype(torch::kInt64));
  const size_t nb = knnag_variant_workspace_bytes(d.B, d.Q, d.P, d.dtype);
  auto ws = scratch(nb, q);
  check_status(knnag_forward_lookup(q.data_ptr(), p.data_ptr(), f.data_ptr(), sigma.data_ptr(), R.data_ptr(),
                                    knn_table.data_ptr<int64_t>(), (int)knn_table.size(1), d.B, d.Q, d.P, d.F, (int)K,
                                    d.dtype, f_out.data_ptr(), w_out.data_ptr(), dists.data_ptr(),
                                    idxs.data_ptr<int64_t>(), ws.data_ptr(), nb, stream_of(q)),
               "knn_lookup_aggregate_aniso_forward");
  return {f_out, w_out, dists, idxs};
}

std::vector<torch::Tensor> knn_aggregate_forward(torch::Tensor q, torch::Tensor p, torch::Tensor f,
                                                 torch::Tensor sigma, int64_t K) {
  KNN_CHECK_INPUT(q);
  KNN_CHECK_INPUT(p);
  KNN_CHECK_INPUT(f);
  KNN_CHECK_INPUT(sigma);
  TORCH_CHECK(q.dim() == 3 && q.size(2) == 3 && p.dim() == 3 && p.size(2) == 3 && p.size(0) == q.size(0),
              "q and p must have shapes [B, Q, 3] and [B, P, 3]");
  const int B = (int)q.size(0), Q = (int)q.size(1), P = (int)p.size(1);
  TORCH_CHECK(f.dim() == 3 && f.size(0) == B && f.size(1) == P, "f must have shape [B, P, F]");
  TORCH_CHECK(sigma.dim() == 3 && sigma.size(0) == B && sigma.size(1) == P && sigma.size(2) >= 1,
              "sigma must have shape [B, P, S] (component 0 is used)");
  const int dt = dtype_code(q);
  for (const torch::Tensor* t : {&p, &f, &sigma})
    TORCH_CHECK(t->scalar_type() == q.scalar_type(), "all floating-point inputs must share q's dtype");
  check_k(K, P);
  const int F = (int)f.size(2);
  const c10::cuda::CUDAGuard guard(q.device());
  auto f_out = torch::empty({B, Q, F}, f.options());
  auto w_out = torch::empty({B, Q, 1}, f.options());
  auto dists = torch::empty({B, Q, K}, q.options());
  auto idxs = torch::empty({B, Q, K}, q.options().dtype(torch::kInt64));
  check_status(knnag_forward_isotropic(q.data_ptr(), p.data_ptr(), f.data_ptr(), sigma.data_ptr(), (int)sigma.size(2),
                                       B, Q, P, F, (int)K, dt, f_out.data_ptr(), w_out.data_ptr(), dists.data_ptr(),
                                       idxs.data_ptr<int64_t>(), stream_of(q)),
               "knn_aggregate_forward");
  return {f_out, w_out, dists, idxs};
}

// --------------------------------------------------------- extended ops

std::vector<torch::Tensor> forward_ex(torch::Tensor q, torch::Tensor p, torch::Tensor f, torch::Tensor sigma,
                                      torch::Tensor R, int64_t K) {
  return forward_impl(q, p, f, sigma, R, K, true);
}

// The adjacency of idxs; `counted` (optional): the buffer a counting
// forward wrote the per-row entry counts into -- it is completed in place.
torch::Tensor build_adjacency_impl(const torch::Tensor& idxs, int64_t P, const torch::Tensor& counted, void* stream) {
  const int B = (int)idxs.size(0), Q = (int)idxs.size(1), K = (int)idxs.size(2);
  check_k(K, (int)P);
  if (counted.defined() && counted.numel() > 0) {
    TORCH_CHECK(counted.is_cuda() && counted.scalar_type() == torch::kUInt8 &&
                    (size_t)counted.numel() >= knnag_adjacency_bytes(B, Q, (int)P, K),
                "counted adjacency must be the uint8 CUDA buffer of a counting forward");
    check_status(knnag_build_adjacency_counted(idxs.data_ptr<int64_t>(), B, Q, (int)P, K, counted.data_ptr(), stream),
                 "build_adjacency");
    return counted;
  }
  auto adj = scratch(knnag_adjacency_bytes(B, Q, (int)P, K), idxs);
  check_status(knnag_build_adjacency(idxs.data_ptr<int64_t>(), B, Q, (int)P, K, adj.data_ptr(), stream),
               "build_adjacency");
  return adj;
}

torch::Tensor build_adjacency(torch::Tensor idxs, int64_t P) {
  KNN_CHECK_INPUT(idxs);
  TORCH_CHECK(idxs.scalar_type() == torch::kInt64 && idxs.dim() == 3, "idxs must be int64 [B, Q, K]");
  const c10::cuda::CUDAGuard guard(idxs.device());
  return build_adjacency_impl(idxs, P, torch::Tensor(), stream_of(idxs));
}

// The same on a pool stream forked from the current one, so that it runs
// beside the next kernels of the current stream.  The buffer is allocated on
// the current stream; the caller must call join.block(current stream)
// before the buffer is used or released there.
torch::Tensor build_adjacency_forked(const torch::Tensor& idxs, int64_t P, at::cuda::CUDAEvent& join,
                                     const torch::Tensor& counted) {
  const int B = (int)idxs.size(0), Q = (int)idxs.size(1), K = (int)idxs.size(2);
  check_k(K, (int)P);
  const c10::cuda::CUDAGuard guard(idxs.device());
  // a fresh buffer is allocated here, on the current stream, before the fork
  const bool use_counted = counted.defined() && counted.numel() > 0;
  torch::Tensor fresh;
  if (!use_counted) fresh = scratch(knnag_adjacency_bytes(B, Q, (int)P, K), idxs);
  const auto dev = idxs.device().index();
  auto main = at::cuda::getCurrentCUDAStream(dev);
  auto side = at::cuda::getStreamFromPool(false, dev);
  at::cuda::CUDAEvent fork;
  fork.record(main);
  fork.block(side);
  torch::Tensor adj = use_counted ? build_adjacency_impl(idxs, P, counted, side.stream()) : fresh;
  if (!use_counted)
    check_status(knnag_build_adjacency(idxs.data_ptr<int64_t>(), B, Q, (int)P, K, adj.data_ptr(), side.stream()),
                 "build_adjacency");
  join.record(side);
  return adj;
}

// rowptr [B*P+1] and sorted entry ids [B*Q*K] views of an adjacency buffer.
std::vector<torch::Tensor> adjacency_views(torch::Tensor adj, int64_t B, int64_t Q, int64_t P, int64_t K) {
  const size_t rows = (size_t)B * P, n = (size_t)B * Q * K;
  // layout: rowptr | cursor | unsorted | entries, each rounded up to 256 bytes
  const size_t a0 = ((rows + 1) * 4 + 255) / 256 * 256;
  const size_t a1 = (rows * 4 + 255) / 256 * 256;
  const size_t a2 = (n * 4 + 255) / 256 * 256;
  auto i32 = adj.view(torch::kInt32);
  auto rowptr = i32.narrow(0, 0, (int64_t)rows + 1);
  auto entries = i32.narrow(0, (int64_t)((a0 + a1 + a2) / 4), (int64_t)n);
  return {rowptr, entries};
}

std::vector<torch::Tensor> backward_ex(torch::Tensor gfo, torch::Tensor q, torch::Tensor p, torch::Tensor f,
                                       torch::Tensor sigma, torch::Tensor R, torch::Tensor idxs,
                                       c10::optional<torch::Tensor> points, c10::optional<torch::Tensor> adjacency,
                                       int64_t needs) {
  return backward_impl(1, c10::nullopt, gfo, q, p, f, sigma, R, c10::nullopt, idxs, points, adjacency, c10::nullopt,
                       needs, true);
}

std::vector<torch::Tensor> backward2_ex(torch::Tensor ggq, torch::Tensor gfo, torch::Tensor q, torch::Tensor p,
                                        torch::Tensor f, torch::Tensor sigma, torch::Tensor R, torch::Tensor idxs,
                                        c10::optional<torch::Tensor> points, c10::optional<torch::Tensor> adjacency,
                                        c10::optional<torch::Tensor> coef, int64_t needs) {
  return backward_impl(2, ggq, gfo, q, p, f, sigma, R, c10::nullopt, idxs, points, adjacency, coef, needs, false);
}

// ------------------------------------------------------------- autograd
//
// The autograd pair of knn_aggregate_aniso (reference
// cuda_knn_aggregate/__init__.py:64-117, 216-289) as C++ Functions.  Inside
// a C++ backward, ctx->needs_input_grad(i) asks the running graph task
// whether input i's gradient is used -- autograd.grad(f_out.sum(), q), the
// first step of an Eikonal loss, uses only dq -- so each order computes only
// the gradients that are used (the point-side kernels and the adjacency are
// skipped when no point gradient is wanted).  Only f_out is differentiable;
// the second order flows only through dq.  Outputs that are not computed are
// zero-size placeholders that are never returned as gradients.

using torch::autograd::AutogradContext;
using torch::autograd::variable_list;

constexpr int64_t kNeedBits[5] = {KNNAG_NEED_DQ, KNNAG_NEED_DP, KNNAG_NEED_DF, KNNAG_NEED_DSIGMA, KNNAG_NEED_DR};
constexpr int64_t kPointBits = KNNAG_NEED_DP | KNNAG_NEED_DF | KNNAG_NEED_DSIGMA | KNNAG_NEED_DR;
// Host-only flag of AggBackwardFn: the graph being built may ask the second
// order for point gradients, so the adjacency is built now, beside the
// first-order kernels (never passed to the C ABI).
constexpr int64_t kPrebuildAdjacency = int64_t(1) << 20;

torch::Tensor or_placeholder(const torch::Tensor& t, const torch::Tensor& like) {
  return t.defined() ? t : torch::empty({0}, like.options());
}

// A gradient that is one value broadcast over its shape (every dimension of
// size > 1 has stride 0) -- what autograd passes for f_out.sum().  It is
// handed to the kernels as that one value instead of being materialised.
bool is_broadcast_scalar(const torch::Tensor& g) {
  if (!g.defined() || g.numel() == 0) return false;
  for (int64_t i = 0; i < g.dim(); ++i)
    if (g.size(i) > 1 && g.stride(i) != 0) return false;
  return true;
}

struct AggBackwardFn : public torch::autograd::Function<AggBackwardFn> {
  // differentiable inputs: gfo, q, p, f, sigma, R; then idxs, points and the
  // adjacency counted by the forward (empty if none) (no grad)
  static variable_list forward(AutogradContext* ctx, torch::Tensor gfo, torch::Tensor q, torch::Tensor p,
                               torch::Tensor f, torch::Tensor sigma, torch::Tensor R, torch::Tensor idxs,
                               torch::Tensor points, torch::Tensor adj_counted, int64_t needs) {
    torch::Tensor adj;
    at::cuda::CUDAEvent join;
    const bool forked = (needs & kPrebuildAdjacency) && !(needs & kPointBits);
    needs &= ~kPrebuildAdjacency;
    if (needs & kPointBits) {
      const c10::cuda::CUDAGuard guard(idxs.device());
      adj = build_adjacency_impl(idxs, p.size(1), adj_counted, stream_of(idxs));
    }
    if (forked) adj = build_adjacency_forked(idxs, p.size(1), join, adj_counted);
    auto o = backward_impl(1, c10::nullopt, gfo, q, p, f, sigma, R, c10::nullopt, idxs, points,
                           (adj.defined() && !forked) ? c10::optional<torch::Tensor>(adj) : c10::nullopt,
                           c10::nullopt, needs, true);
    if (forked) join.block(at::cuda::getCurrentCUDAStream(q.device().index()));
    ctx->save_for_backward({gfo, q, p, f, sigma, R, idxs, points});
    ctx->saved_data["coef"] = o[5];
    ctx->saved_data["gfo_scalar"] = (needs & KNNAG_GFO_SCALAR) != 0;
    if (adj.defined()) ctx->saved_data["adj"] = adj;
    ctx->set_materialize_grads(false);
    return {or_placeholder(o[0], q), or_placeholder(o[1], q), or_placeholder(o[2], q), or_placeholder(o[3], q),
            or_placeholder(o[4], q)};
  }

  static variable_list backward(AutogradContext* ctx, variable_list gg) {
    variable_list out(10);
    if (gg.empty() || !gg[0].defined()) return out;  // only dq is differentiated
    int64_t needs = 0;
    if (ctx->needs_input_grad(0)) needs |= KNNAG_NEED_DGFO;
    for (int i = 0; i < 5; ++i)
      if (ctx->needs_input_grad(1 + i)) needs |= kNeedBits[i];
    if (!needs) return out;
    if (ctx->saved_data["gfo_scalar"].toBool()) needs |= KNNAG_GFO_SCALAR;
    auto s = ctx->get_saved_variables();
    torch::Tensor adj;
    if (ctx->saved_data.count("adj")) adj = ctx->saved_data["adj"].toTensor();
    if ((needs & kPointBits) && !adj.defined()) adj = build_adjacency(s[6], s[2].size(1));
    auto o = backward_impl(2, gg[0].contiguous(), s[0], s[1], s[2], s[3], s[4], s[5], c10::nullopt, s[6], s[7],
                           adj.defined() ? c10::optional<torch::Tensor>(adj) : c10::nullopt,
                           ctx->saved_data["coef"].toTensor(), needs, false);
    for (int i = 0; i < 6; ++i) out[i] = o[i];
    return out;
  }
};

struct AggFn : public torch::autograd::Function<AggFn> {
  static variable_list forward(AutogradContext* ctx, torch::Tensor q, torch::Tensor p, torch::Tensor f,
                               torch::Tensor sigma, torch::Tensor R, int64_t K) {
    // a point input that requires grad: its backward will want the
    // adjacency, whose first pass (row counts) the forward makes for free
    const bool want_adj = p.requires_grad() || f.requires_grad() || sigma.requires_grad() || R.requires_grad();
    auto o = forward_impl(q, p, f, sigma, R, K, true, want_adj);
    ctx->save_for_backward({q, p, f, sigma, R, o[3]});
    ctx->saved_data["points"] = o[4];
    if (want_adj) ctx->saved_data["adj_counted"] = o[5];
    ctx->set_materialize_grads(false);
    return {o[0], o[1], o[2], o[3]};
  }

  static variable_list backward(AutogradContext* ctx, variable_list g) {
    variable_list out(6);
    if (g.empty() || !g[0].defined()) return out;  // grad_w_out / grad_dists are not propagated
    int64_t needs = 0;
    for (int i = 0; i < 5; ++i)
      if (ctx->needs_input_grad(i)) needs |= kNeedBits[i];
    if (!needs) return out;
    auto s = ctx->get_saved_variables();
    const bool scalar = is_broadcast_scalar(g[0]);
    // create_graph with point inputs that require grad: the second order of
    // this graph may want point gradients (the Eikonal step does)
    const bool prebuild = torch::GradMode::is_enabled() &&
                          (s[1].requires_grad() || s[2].requires_grad() || s[3].requires_grad() || s[4].requires_grad());
    torch::Tensor counted;
    if (ctx->saved_data.count("adj_counted")) counted = ctx->saved_data["adj_counted"].toTensor();
    auto r = AggBackwardFn::apply(scalar ? g[0] : g[0].contiguous(), s[0], s[1], s[2], s[3], s[4], s[5],
                                  ctx->saved_data["points"].toTensor(), or_placeholder(counted, s[5]),
                                  needs | (scalar ? KNNAG_GFO_SCALAR : 0) | (prebuild ? kPrebuildAdjacency : 0));
    for (int i = 0; i < 5; ++i) out[i] = (needs & kNeedBits[i]) ? r[i] : torch::Tensor();
    return out;
  }
};

std::vector<torch::Tensor> knn_aggregate_aniso_autograd(torch::Tensor q, torch::Tensor p, torch::Tensor f,
                                                        torch::Tensor sigma, torch::Tensor R, int64_t K) {
  return AggFn::apply(q, p, f, sigma, R, K);
}

}  // namespace

PYBIND11_MODULE(_C, m) {
  m.def("knn_aggregate_aniso_forward", &knn_aggregate_aniso_forward, "KNN aggregate aniso forward");
  m.def("knn_aggregate_aniso_backward", &knn_aggregate_aniso_backward, "KNN aggregate aniso backward");
  m.def("knn_aggregate_aniso_backward_2nd", &knn_aggregate_aniso_backward_2nd,
        "KNN aggregate aniso second order backward");
  m.def("knn_aggregate_forward", &knn_aggregate_forward, "KNN aggregate forward");
  m.def("knn_lookup_aggregate_aniso_forward", &knn_lookup_aggregate_aniso_forward, "KNN lookup aggregate aniso forward");
  m.def("knn_precomputed_aggregate_aniso_forward", &knn_precomputed_aggregate_aniso_forward,
        "KNN precomputed aggregate aniso forward");
  m.def("forward_ex", &forward_ex, "forward that also returns the packed point records");
  m.def("knn_aggregate_aniso_autograd", &knn_aggregate_aniso_autograd,
        "differentiable forward (C++ autograd Functions; gradients computed only where the graph task uses them)");
  m.def("build_adjacency", &build_adjacency, "point -> entry adjacency (CSR) of idxs");
  m.def("adjacency_views", &adjacency_views, "rowptr / entry views of an adjacency buffer");
  m.def("backward_ex", &backward_ex, "first-order adjoint with selectable outputs; also returns coef");
  m.def("backward2_ex", &backward2_ex, "second-order adjoint with selectable outputs");
  m.attr("NEED_DQ") = (int)KNNAG_NEED_DQ;
  m.attr("NEED_DP") = (int)KNNAG_NEED_DP;
  m.attr("NEED_DF") = (int)KNNAG_NEED_DF;
  m.attr("NEED_DSIGMA") = (int)KNNAG_NEED_DSIGMA;
  m.attr("NEED_DR") = (int)KNNAG_NEED_DR;
  m.attr("NEED_DGFO") = (int)KNNAG_NEED_DGFO;
}
