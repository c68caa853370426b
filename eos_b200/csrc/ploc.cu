// PLOC hierarchy: parallel locally-ordered clustering (Meister & Bittner, "Parallel Locally-
// Ordered Clustering for Bounding Volume Hierarchy Construction", IEEE TVCG 2018), a second
// builder beside the Karras LBVH.  No reference counterpart (the reference builds a CPU
// SAH tree, src/BVH.cpp:97-111); it is a tree-quality choice only -- the traversal's
// results do not depend on the tree.
//
// Input: the leaf boxes in Morton order.  Clusters start as the leaves; each iteration
//   1. every cluster finds its nearest neighbour among the clusters within kRadius places
//      of it (distance = surface area of the merged box; ties to the lower index);
//   2. mutual nearest neighbours merge into a new interior node at the lower position;
//   3. the surviving clusters are compacted in order.
// Interior nodes are numbered in creation order (deterministic: one exclusive scan of
// packed keep / make flags per round, no atomics), the root last.  Afterwards every node's first leaf position in depth-first
// order (left subtree first) is found by a walk to the root, so that every subtree covers
// a contiguous range of triangle records; the nodes are renumbered root-first into the
// layout the refit and the node-record writer expect (interior 0..n-2 with the root 0,
// leaf at position q -> n-1+q).
#include <algorithm>
#include <vector>


#include "eos_internal.cuh"
#include "scan.cuh"

namespace eos {
namespace {

constexpr int kRadius = 16;        // neighbours searched on each side
constexpr int kNNBlock = 256;
constexpr int kTail = 1024;  // clusters at or below which one block runs the remaining rounds
constexpr int kMaxWalk = 4 * kStackMax;  // bound of the walks to the root

__device__ __forceinline__ float merged_area(float4 al, float4 ah, float4 bl, float4 bh) {
  const float dx = fmaxf(ah.x, bh.x) - fminf(al.x, bl.x);
  const float dy = fmaxf(ah.y, bh.y) - fminf(al.y, bl.y);
  const float dz = fmaxf(ah.z, bh.z) - fminf(al.z, bl.z);
  return dx * dy + dy * dz + dz * dx;
}

// Leaf p's node id in the refit's numbering (n - 1 + p): the initial clusters.
__global__ void k_ploc_leaf_ids(int n, int* __restrict__ cid) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) cid[p] = n - 1 + p;
}

// Nearest neighbour of every cluster within kRadius places (boxes staged in shared memory).
__global__ void k_ploc_nn(const int* __restrict__ state, const float4* __restrict__ lo, const float4* __restrict__ hi,
                          int* __restrict__ nn) {
  __shared__ float4 slo[kNNBlock + 2 * kRadius], shi[kNNBlock + 2 * kRadius];
  const int nc = state[0];
  const int b0 = blockIdx.x * kNNBlock;
  for (int t = threadIdx.x; t < kNNBlock + 2 * kRadius; t += blockDim.x) {
    const int g = b0 - kRadius + t;
    if (g >= 0 && g < nc) {
      slo[t] = lo[g];
      shi[t] = hi[g];
    }
  }
  __syncthreads();
  const int i = b0 + threadIdx.x;
  if (i >= nc) return;
  const int li = threadIdx.x + kRadius;
  const float4 al = slo[li], ah = shi[li];
  float best = kInf;
  int bj = i == 0 ? 1 : i - 1;
  const int j0 = max(0, i - kRadius), j1 = min(nc - 1, i + kRadius);
  for (int j = j0; j <= j1; ++j) {
    if (j == i) continue;
    const int lj = j - b0 + kRadius;
    const float a = merged_area(al, ah, slo[lj], shi[lj]);
    if (a < best) {
      best = a;
      bj = j;
    }
  }
  nn[i] = bj;
}

// Cluster i survives (keep) unless it is the upper half of a mutual pair; the lower half
// of a pair creates a node (make).  With `force` (an iteration that merged nothing) the
// pairs (2k, 2k + 1) merge instead, which bounds the number of iterations.
// keep in the low 32 bits, make in the high 32 bits: one scan counts both.
// The scan runs over nc_ub + 1 entries (nc_ub: the host's upper bound of nc); the entries
// from nc on are 0, so the scan's value at nc is the round's total.  Each block of
// kScanBlock entries also writes its sum to bsum (the scan's first step, scan.cuh).
__global__ void __launch_bounds__(kScanBlock) k_ploc_flags(const int* __restrict__ state, int nc_ub,
                                                           const int* __restrict__ nn, int force,
                                                           unsigned long long* __restrict__ km,
                                                           unsigned long long* __restrict__ bsum) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = state[0];
  unsigned long long v = 0ull;
  if (i < nc) {
    int partner;
    if (force) {
      partner = (i & 1) ? i - 1 : (i + 1 < nc ? i + 1 : -1);
    } else {
      const int j = nn[i];
      partner = (j >= 0 && j < nc && nn[j] == i) ? j : -1;
    }
    const unsigned long long keep = partner < 0 || i < partner;
    const unsigned long long make = partner >= 0 && i < partner;
    v = keep | (make << 32);
  }
  if (i <= nc_ub) km[i] = v;
  block_total(v, bsum);
}

// Also writes the next round's state (clusters kept, nodes made so far, nodes made by this
// round) to state_out and to the host's read-back slot.  The exclusive scan of km is this
// block's scan of its entries plus the block's scanned sum (bsum after k_scan_totals;
// bsum[n_blocks] = the round's total); same grid as k_ploc_flags.
__global__ void __launch_bounds__(kScanBlock) k_ploc_merge(
    const int* __restrict__ state, int* __restrict__ state_out, int* __restrict__ slot, const int* __restrict__ nn,
    int force, int nc_ub, const unsigned long long* __restrict__ km, const unsigned long long* __restrict__ bsum,
    int n_blocks, const int* __restrict__ cid, const float4* __restrict__ lo, const float4* __restrict__ hi,
    int* __restrict__ cid_out, float4* __restrict__ lo_out, float4* __restrict__ hi_out, int2* __restrict__ child,
    int* __restrict__ count, float4* __restrict__ nlo, float4* __restrict__ nhi, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = state[0], node_base = state[1];
  unsigned long long block_sum;
  const unsigned long long sc = bsum[blockIdx.x] + block_exclusive_scan(i <= nc_ub ? km[i] : 0ull, block_sum);
  if (i >= nc) return;
  if (i == 0) {
    const unsigned long long total = bsum[n_blocks];
    const int kept = (int)(total & 0xffffffffull), made = (int)(total >> 32);
    state_out[0] = slot[0] = kept;
    state_out[1] = slot[1] = node_base + made;
    state_out[2] = slot[2] = made;
  }
  int partner;
  if (force) {
    partner = (i & 1) ? i - 1 : (i + 1 < nc ? i + 1 : -1);
  } else {
    const int j = nn[i];
    partner = (j >= 0 && j < nc && nn[j] == i) ? j : -1;
  }
  if (partner >= 0 && i > partner) return;  // merged into the lower cluster
  const int pos = (int)(sc & 0xffffffffull);
  if (partner < 0) {
    cid_out[pos] = cid[i];
    lo_out[pos] = lo[i];
    hi_out[pos] = hi[i];
    return;
  }
  const int k = node_base + (int)(sc >> 32);
  const int a = cid[i], b = cid[partner];
  const float4 al = lo[i], ah = hi[i], bl = lo[partner], bh = hi[partner];
  const float4 l = make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), 0.0f);
  const float4 h = make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), 0.0f);
  child[k] = make_int2(a, b);
  count[k] = (a >= n - 1 ? 1 : count[a]) + (b >= n - 1 ? 1 : count[b]);
  nlo[k] = l;
  nhi[k] = h;
  cid_out[pos] = k;
  lo_out[pos] = l;
  hi_out[pos] = h;
}

// Round state on the device: [0] clusters, [1] interior nodes made so far, [2] nodes made
// by the last round.  Rounds are launched ahead of the host, which reads the state back a
// few rounds later (build_ploc).
__global__ void k_ploc_state_init(int* __restrict__ state, int n) {
  state[0] = n;
  state[1] = 0;
  state[2] = 1;
}

// The rounds left once at most kTail clusters remain, in one block with the clusters in
// shared memory: the same neighbour search, pair rule, forced round after a round that
// merged nothing, and creation-order numbering as the per-round kernels, so the tree is
// the same; what it saves is the launches of the last ~30 rounds.
__global__ void __launch_bounds__(kTail) k_ploc_tail(int* __restrict__ state, const int* __restrict__ cid_in,
                                                     const float4* __restrict__ lo_in, const float4* __restrict__ hi_in,
                                                     int2* __restrict__ child, int* __restrict__ count,
                                                     float4* __restrict__ nlo, float4* __restrict__ nhi, int n,
                                                     int* __restrict__ err) {
  __shared__ float4 slo[kTail], shi[kTail];
  __shared__ int scid[kTail], snn[kTail];
  __shared__ int wsum[kTail / 32];
  const int i = threadIdx.x, lane = i & 31, warp = i >> 5;
  int nc = state[0], node_base = state[1];
  int force = state[2] == 0 && nc > 1;  // the last round merged nothing: the forced round is next
  if (nc > kTail) {  // the host launches this only at or below kTail
    if (i == 0) atomicOr(err, kErrIndex);
    return;
  }
  if (i < nc) {
    slo[i] = lo_in[i];
    shi[i] = hi_in[i];
    scid[i] = cid_in[i];
  }
  __syncthreads();
  int made = 1, iters = 0;
  while (nc > 1) {
    if (++iters > 4 * kTail + 8) {  // cannot happen: every round or its forced repeat merges
      if (i == 0) atomicOr(err, kErrTimeout);
      break;
    }
    if (!force && i < nc) {
      const float4 al = slo[i], ah = shi[i];
      float best = kInf;
      int bj = i == 0 ? 1 : i - 1;
      const int j0 = max(0, i - kRadius), j1 = min(nc - 1, i + kRadius);
      for (int j = j0; j <= j1; ++j) {
        if (j == i) continue;
        const float a = merged_area(al, ah, slo[j], shi[j]);
        if (a < best) {
          best = a;
          bj = j;
        }
      }
      snn[i] = bj;
    }
    __syncthreads();
    int partner = -1;
    if (i < nc) {
      if (force) {
        partner = (i & 1) ? i - 1 : (i + 1 < nc ? i + 1 : -1);
      } else {
        const int j = snn[i];
        partner = (j >= 0 && j < nc && snn[j] == i) ? j : -1;
      }
    }
    const int keep = i < nc && (partner < 0 || i < partner);
    const int make = i < nc && partner >= 0 && i < partner;
    // block exclusive scan of keep (low 16 bits) and make (high 16 bits)
    const int v = keep | (make << 16);
    int inc = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= d) inc += u;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < kTail / 32; ++w) {
      const int t = wsum[w];
      before += w < warp ? t : 0;
      total += t;
    }
    const int ex = before + inc - v;
    const int pos = ex & 0xffff, mk = ex >> 16;
    const int kept = total & 0xffff;
    made = total >> 16;
    int out_id = 0;
    float4 ol = make_float4(0.0f, 0.0f, 0.0f, 0.0f), oh = ol;
    if (keep) {
      if (partner < 0) {
        out_id = scid[i];
        ol = slo[i];
        oh = shi[i];
      } else {
        const int k = node_base + mk;
        const int a = scid[i], b = scid[partner];
        const float4 al = slo[i], ah = shi[i], bl = slo[partner], bh = shi[partner];
        ol = make_float4(fminf(al.x, bl.x), fminf(al.y, bl.y), fminf(al.z, bl.z), 0.0f);
        oh = make_float4(fmaxf(ah.x, bh.x), fmaxf(ah.y, bh.y), fmaxf(ah.z, bh.z), 0.0f);
        child[k] = make_int2(a, b);
        count[k] = (a >= n - 1 ? 1 : count[a]) + (b >= n - 1 ? 1 : count[b]);
        nlo[k] = ol;
        nhi[k] = oh;
        out_id = k;
      }
    }
    __syncthreads();  // every read of this round's clusters is done
    if (keep) {
      scid[pos] = out_id;
      slo[pos] = ol;
      shi[pos] = oh;
    }
    __syncthreads();
    node_base += made;
    nc = kept;
    force = made == 0 && !force;
  }
  if (i == 0) {
    state[0] = nc;
    state[1] = node_base;
    state[2] = made;
  }
}

__global__ void k_ploc_parents(int n, const int2* __restrict__ child, int* __restrict__ parent) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n - 1) return;
  const int2 c = child[k];
  parent[c.x] = k;
  parent[c.y] = k;
}

// Depth-first position of the first leaf of every node (creation-order ids: interior
// 0..n-2, root n-2; leaf Morton position p -> n-1+p): the sum of the left siblings' leaf
// counts along the path to the root.
__global__ void k_ploc_positions(int n, const int2* __restrict__ child, const int* __restrict__ parent,
                                 const int* __restrict__ count, int* __restrict__ first, int* __restrict__ depth_max) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= 2 * n - 1) return;
  int pos = 0, node = v, steps = 0;
  while (node != n - 2) {
    const int p = parent[node];
    if (p < 0 || ++steps > kMaxWalk) {  // reported as too deep: the caller falls back to the LBVH
      atomicMax(depth_max, kMaxWalk + 1);
      return;
    }
    const int2 c = child[p];
    if (c.y == node) pos += c.x >= n - 1 ? 1 : count[c.x];
    node = p;
  }
  first[v] = pos;
  atomicMax(depth_max, steps);
}

// Root-first renumbering into the refit's layout; perm[p] = final position of the leaf at
// Morton position p.
__global__ void k_ploc_finalize(int n, const int2* __restrict__ child, const int* __restrict__ count,
                                const int* __restrict__ first, int2* __restrict__ child_out,
                                int2* __restrict__ range_out, int* __restrict__ parent_out, uint32_t* __restrict__ perm) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) perm[k] = (uint32_t)first[n - 1 + k];
  if (k >= n - 1) return;
  auto map = [&](int x) { return x >= n - 1 ? n - 1 + first[x] : n - 2 - x; };
  const int f = n - 2 - k;
  const int2 c = child[k];
  const int a = map(c.x), b = map(c.y);
  child_out[f] = make_int2(a, b);
  range_out[f] = make_int2(first[k], first[k] + count[k] - 1);
  parent_out[a] = f;
  parent_out[b] = f;
}

inline int grid_of(long long n, int block) { return (int)std::max<long long>(1, (n + block - 1) / block); }

}  // namespace

// Builds the hierarchy over n >= 2 leaves whose boxes lie at blo / bhi[n-1+p] (Morton
// position p).  Writes child / range / parent in the refit's layout and perm[p], the final
// record position of Morton position p.  *depth = the deepest node's depth; above
// 4 * kStackMax nothing is written and the caller must use another builder.
eos_status build_ploc(eos_ctx* ctx, int n, const float4* blo, const float4* bhi, int2* child, int2* range,
                      int* parent, uint32_t* perm, int* depth) {
  cudaStream_t st = ctx->stream;
  eos_status es = EOS_OK;
  const size_t nn = (size_t)n;
  int* cid[2] = {(int*)scratch(ctx, "ploc.cid0", 4 * nn, &es), (int*)scratch(ctx, "ploc.cid1", 4 * nn, &es)};
  float4* clo[2] = {(float4*)scratch(ctx, "ploc.lo0", 16 * nn, &es), (float4*)scratch(ctx, "ploc.lo1", 16 * nn, &es)};
  float4* chi[2] = {(float4*)scratch(ctx, "ploc.hi0", 16 * nn, &es), (float4*)scratch(ctx, "ploc.hi1", 16 * nn, &es)};
  int* nbr = (int*)scratch(ctx, "ploc.nn", 4 * nn, &es);
  unsigned long long* km = (unsigned long long*)scratch(ctx, "ploc.km", 8 * (nn + 1), &es);
  unsigned long long* bsum = (unsigned long long*)scratch(ctx, "ploc.bsum", 8 * ((size_t)scan_blocks(n + 1) + 1), &es);
  int2* tchild = (int2*)scratch(ctx, "ploc.child", 8 * nn, &es);
  int* tcount = (int*)scratch(ctx, "ploc.count", 4 * nn, &es);
  float4* tlo = (float4*)scratch(ctx, "ploc.nlo", 16 * nn, &es);
  float4* thi = (float4*)scratch(ctx, "ploc.nhi", 16 * nn, &es);
  int* tparent = (int*)scratch(ctx, "ploc.parent", 4 * (2 * nn), &es);
  int* first = (int*)scratch(ctx, "ploc.first", 4 * (2 * nn), &es);
  int* dmax = (int*)scratch(ctx, "ploc.depth", 4, &es);
  if (es != EOS_OK) return es;

  // clusters = leaves in Morton order
  EOS_CUDA(cudaMemcpyAsync(clo[0], blo + (n - 1), 16 * nn, cudaMemcpyDeviceToDevice, st));
  EOS_CUDA(cudaMemcpyAsync(chi[0], bhi + (n - 1), 16 * nn, cudaMemcpyDeviceToDevice, st));
  k_ploc_leaf_ids<<<grid_of(n, 256), 256, 0, st>>>(n, cid[0]);
  // Rounds run ahead of the host until at most kTail clusters are left (k_ploc_tail does the
  // rest): grids are sized by an upper bound of the cluster count
  // (the last one read back; it only falls), and the host reads each round's state
  // kAhead rounds later instead of waiting after every round.  A round that merges nothing
  // changes nothing, so the rounds queued behind one repeat it harmlessly; when the host
  // sees it, it waits for the queue and runs the forced round (as a synchronous loop
  // would right away), so the tree is the same.
  constexpr int kAhead = 4;
  static_assert(kAhead <= (int)(sizeof(ctx->ring_ev) / sizeof(ctx->ring_ev[0])), "one event per slot");
  int* state = (int*)scratch(ctx, "ploc.state", 32, &es);  // two states, by round parity
  if (es != EOS_OK) return es;
  if (!ctx->ring_host) {
    if (cudaHostAlloc(&ctx->ring_host, 16 * kAhead, cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(&ctx->ring_dev, ctx->ring_host, 0) != cudaSuccess) {
      cudaGetLastError();
      if (ctx->ring_host) cudaFreeHost(ctx->ring_host);
      ctx->ring_host = ctx->ring_dev = nullptr;
      return EOS_ERR_OOM;
    }
  }
  for (cudaEvent_t& e : ctx->ring_ev)
    if (!e) EOS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  volatile int* snap = ctx->ring_host;
  k_ploc_state_init<<<1, 1, 0, st>>>(state, n);
  int nc_ub = n, cur = 0;
  long long issued = 0, read = 0;
  auto enqueue = [&](int force) {
    if (!force) k_ploc_nn<<<grid_of(nc_ub, kNNBlock), kNNBlock, 0, st>>>(state + 4 * cur, clo[cur], chi[cur], nbr);
    const int nb = scan_blocks(nc_ub + 1);
    k_ploc_flags<<<nb, kScanBlock, 0, st>>>(state + 4 * cur, nc_ub, nbr, force, km, bsum);
    k_scan_totals<<<1, 1024, 0, st>>>(bsum, nb);
    const int slot = (int)(issued % kAhead);
    k_ploc_merge<<<nb, kScanBlock, 0, st>>>(state + 4 * cur, state + 4 * (cur ^ 1), ctx->ring_dev + 4 * slot, nbr,
                                            force, nc_ub, km, bsum, nb, cid[cur], clo[cur], chi[cur], cid[cur ^ 1],
                                            clo[cur ^ 1], chi[cur ^ 1], tchild, tcount, tlo, thi, n);
    if (cudaGetLastError() != cudaSuccess) return false;
    if (cudaEventRecord(ctx->ring_ev[slot], st) != cudaSuccess) return false;
    cur ^= 1;
    ++issued;
    return true;
  };
  bool ok = true;
  for (;;) {
    if (issued - read == kAhead || !ok) {  // read the oldest round in flight
      const int slot = (int)(read % kAhead);
      if (!ok || cudaEventSynchronize(ctx->ring_ev[slot]) != cudaSuccess) return EOS_ERR_CUDA;
      ++read;
      const int nc = snap[4 * slot], made = snap[4 * slot + 2];
      nc_ub = std::min(nc_ub, nc);
      if (nc <= 1) break;
      if (made == 0) {  // stalled: drain, then the forced round
        EOS_CUDA(cudaStreamSynchronize(st));
        if (!enqueue(1)) return EOS_ERR_CUDA;
        EOS_CUDA(cudaStreamSynchronize(st));
        read = issued;
        nc_ub = std::min(nc_ub, (int)snap[4 * (int)((issued - 1) % kAhead)]);
        if (nc_ub <= 1) break;
      }
    }
    if (nc_ub <= kTail) {  // the rest in one block, behind the rounds in flight
      k_ploc_tail<<<1, kTail, 0, st>>>(state + 4 * cur, cid[cur], clo[cur], chi[cur], tchild, tcount, tlo, thi, n,
                                       ctx->d_err);
      break;
    }
    if (issued > 4ll * n + 8) return EOS_ERR_TIMEOUT;  // cannot happen: every round or its forced repeat merges
    ok = enqueue(0);
  }
  int final_state[4] = {0, 0, 0, 0};
  EOS_CUDA(cudaMemcpyAsync(final_state, state + 4 * cur, 16, cudaMemcpyDeviceToHost, st));
  EOS_CUDA(cudaStreamSynchronize(st));
  const int node_base = final_state[1];
  if (node_base != n - 1) return EOS_ERR_CUDA;
  EOS_CUDA(cudaMemsetAsync(tparent, 0xff, 4 * (2 * nn), st));
  EOS_CUDA(cudaMemsetAsync(dmax, 0, 4, st));
  k_ploc_parents<<<grid_of(n - 1, 256), 256, 0, st>>>(n, tchild, tparent);
  k_ploc_positions<<<grid_of(2 * (long long)n - 1, 256), 256, 0, st>>>(n, tchild, tparent, tcount, first, dmax);
  EOS_CUDA(cudaMemcpyAsync(depth, dmax, 4, cudaMemcpyDeviceToHost, st));
  EOS_CUDA(cudaStreamSynchronize(st));
  if (*depth > kMaxWalk) return EOS_OK;  // some walk did not end: outputs left unwritten
  EOS_CUDA(cudaMemsetAsync(parent, 0xff, 4 * (2 * nn), st));
  k_ploc_finalize<<<grid_of(n, 256), 256, 0, st>>>(n, tchild, tcount, first, child, range, parent, perm);
  return EOS_OK;
}

}  // namespace eos
