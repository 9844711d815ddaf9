// Kernel bodies and how they are launched: one context at a time, or one launch for many.
//
// Every stencil and pointwise kernel of a stage is written as a struct K whose static
// device function K::run(blockIdx, gridDim, args...) is the kernel body; its first two
// parameters shadow CUDA's built-ins, so the body reads its block coordinates from them.
// launch<K>(ctx, grid, block, smem, stream, args...) then either
//   - launches k_one<K> with the built-in coordinates (the ordinary path), or
//   - when the context records (ctx->rec, set by an ensemble while it plans a step),
//     stores the launch: its grid, its block shape and its arguments.
// An ensemble turns the recorded launches of its members into ONE launch of k_many<K> per
// sub-step: the grid is the members' grids laid end to end, a table maps each block to its
// member and to the block's coordinates in that member's own grid, and the member's
// arguments come from a device table.  The kernel body is the same code either way.
#pragma once

#include <cuda/std/tuple>

#include <cstring>
#include <vector>

#include "imex_internal.h"

namespace imex {

// the parameters of a kernel body that stand for the built-in block index and grid shape
#define IMEX_BLK const uint3 blockIdx, const dim3 gridDim
// launch bounds of a body: threads per block (0: none declared) and blocks per SM (0: none)
#define IMEX_BOUNDS(nt, minb) static constexpr int kNT = nt, kMinB = minb;

template <class K, class... A>
__global__ void k_one(A... a) {
  K::run(blockIdx, gridDim, a...);
}
template <class K, class... A>
__global__ void __launch_bounds__(K::kNT) k_one_b(A... a) {
  K::run(blockIdx, gridDim, a...);
}
template <class K, class... A>
__global__ void __launch_bounds__(K::kNT, K::kMinB) k_one_bm(A... a) {
  K::run(blockIdx, gridDim, a...);
}

// device tables of a batched launch: member of each block, first block of each member,
// each member's grid (x, y) and arguments
template <class... A>
struct ManyTab {
  const cuda::std::tuple<A...>* args;
  const int* member;
  const int* first;
  const uint2* grid;
};
template <class K, class... A>
__device__ __forceinline__ void many_body(const ManyTab<A...>& t) {
  const int m = __ldg(t.member + blockIdx.x);
  const int l = (int)blockIdx.x - __ldg(t.first + m);
  const uint2 g = t.grid[m];
  const uint3 b = make_uint3((unsigned)l % g.x, (unsigned)l / g.x, 0u);
  const dim3 gd(g.x, g.y, 1);
  cuda::std::apply([&](const A&... a) { K::run(b, gd, a...); }, t.args[m]);
}
template <class K, class... A>
__global__ void k_many(ManyTab<A...> t) {
  many_body<K, A...>(t);
}
template <class K, class... A>
__global__ void __launch_bounds__(K::kNT) k_many_b(ManyTab<A...> t) {
  many_body<K, A...>(t);
}
template <class K, class... A>
__global__ void __launch_bounds__(K::kNT, K::kMinB) k_many_bm(ManyTab<A...> t) {
  many_body<K, A...>(t);
}

// device-to-device copies of several members in one launch (blockIdx.y = copy)
struct CopyDesc {
  double* dst;
  const double* src;
  long long n;  // doubles
};
__global__ void k_copies(const CopyDesc* __restrict__ d);

// ------------------------------------------------------------------ recording (host)
struct PlanItem;
struct PlanArena {
  std::vector<void*> dev;  // device tables, freed with the plan
};
// One recorded stream operation of a member: a kernel launch, or a device-to-device copy.
struct RecOp {
  // builds the batched launch of ops that share this kernel (same K and argument types)
  imex_status (*plan)(const std::vector<const RecOp*>& ops, PlanArena& arena, PlanItem& item, std::string& err) =
      nullptr;
  dim3 grid;
  unsigned block = 0;
  size_t smem = 0;
  std::vector<unsigned char> args;  // the cuda::std::tuple of the arguments, as bytes
  CopyDesc copy{};                  // plan == nullptr: a copy
};
struct Recorder {
  std::vector<RecOp> ops;
};
// One launch of an ensemble's planned step.
struct PlanItem {
  cudaError_t (*launch)(const PlanItem& it, cudaStream_t s) = nullptr;
  const void* args = nullptr;
  const int* member = nullptr;
  const int* first = nullptr;
  const uint2* grid = nullptr;
  unsigned nblocks = 0, block = 0, gy = 1;
  size_t smem = 0;
  int solve = -1;  // >= 0: a batched solve (BATCH_MAGNETIC / BATCH_PRESSURE) instead of a kernel
};

template <class K, class... A>
cudaError_t launch_many(const PlanItem& it, cudaStream_t s) {
  ManyTab<A...> t{static_cast<const cuda::std::tuple<A...>*>(it.args), it.member, it.first, it.grid};
  if constexpr (K::kNT == 0)
    k_many<K, A...><<<it.nblocks, it.block, it.smem, s>>>(t);
  else if constexpr (K::kMinB == 0)
    k_many_b<K, A...><<<it.nblocks, it.block, it.smem, s>>>(t);
  else
    k_many_bm<K, A...><<<it.nblocks, it.block, it.smem, s>>>(t);
  return cudaGetLastError();
}

imex_status plan_alloc(PlanArena& arena, size_t bytes, void** p, std::string& err);
imex_status plan_upload(void* dst, const void* src, size_t bytes, std::string& err);

template <class K, class... A>
imex_status plan_kernel(const std::vector<const RecOp*>& ops, PlanArena& arena, PlanItem& item, std::string& err) {
  using Tup = cuda::std::tuple<A...>;
  const size_t n = ops.size();
  std::vector<int> first(n), member;
  std::vector<uint2> grid(n);
  std::vector<unsigned char> args(n * sizeof(Tup));
  unsigned total = 0;
  for (size_t m = 0; m < n; ++m) {
    const RecOp& o = *ops[m];
    if (o.block != ops[0]->block || o.smem != ops[0]->smem || o.grid.z != 1) {
      err = "batched launch: members differ in block shape or shared memory";
      return IMEX_ERR_UNSUPPORTED;
    }
    first[m] = (int)total;
    grid[m] = make_uint2(o.grid.x, o.grid.y);
    const unsigned nb = o.grid.x * o.grid.y;
    for (unsigned q = 0; q < nb; ++q) member.push_back((int)m);
    total += nb;
    std::memcpy(args.data() + m * sizeof(Tup), o.args.data(), sizeof(Tup));
  }
  void *d_args, *d_member, *d_first, *d_grid;
  imex_status s;
  if ((s = plan_alloc(arena, args.size(), &d_args, err)) != IMEX_OK ||
      (s = plan_alloc(arena, member.size() * sizeof(int), &d_member, err)) != IMEX_OK ||
      (s = plan_alloc(arena, n * sizeof(int), &d_first, err)) != IMEX_OK ||
      (s = plan_alloc(arena, n * sizeof(uint2), &d_grid, err)) != IMEX_OK)
    return s;
  if ((s = plan_upload(d_args, args.data(), args.size(), err)) != IMEX_OK ||
      (s = plan_upload(d_member, member.data(), member.size() * sizeof(int), err)) != IMEX_OK ||
      (s = plan_upload(d_first, first.data(), n * sizeof(int), err)) != IMEX_OK ||
      (s = plan_upload(d_grid, grid.data(), n * sizeof(uint2), err)) != IMEX_OK)
    return s;
  item.launch = &launch_many<K, A...>;
  item.args = d_args;
  item.member = static_cast<const int*>(d_member);
  item.first = static_cast<const int*>(d_first);
  item.grid = static_cast<const uint2*>(d_grid);
  item.nblocks = total;
  item.block = ops[0]->block;
  item.smem = ops[0]->smem;
  return IMEX_OK;
}

// Launch body K over `grid` (or record the launch when the context records).
template <class K, class... A>
void launch(imex_ctx* ctx, dim3 grid, unsigned block, size_t smem, cudaStream_t s, A... a) {
  if (ctx->rec) {
    using Tup = cuda::std::tuple<A...>;
    RecOp op;
    op.plan = &plan_kernel<K, A...>;
    op.grid = grid;
    op.block = block;
    op.smem = smem;
    Tup t(a...);
    op.args.resize(sizeof(Tup));
    std::memcpy(op.args.data(), &t, sizeof(Tup));
    ctx->rec->ops.push_back(std::move(op));
    return;
  }
  if constexpr (K::kNT == 0)
    k_one<K, A...><<<grid, block, smem, s>>>(a...);
  else if constexpr (K::kMinB == 0)
    k_one_b<K, A...><<<grid, block, smem, s>>>(a...);
  else
    k_one_bm<K, A...><<<grid, block, smem, s>>>(a...);
}

// cudaMemcpyAsync of `n` doubles device to device (or a recorded copy)
cudaError_t copy_d2d(imex_ctx* ctx, double* dst, const double* src, long long n);

}  // namespace imex
