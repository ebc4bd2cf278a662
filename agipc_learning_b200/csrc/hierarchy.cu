// hierarchy.cu -- MAS aggregation hierarchy on the GPU, for the 32-slot bank
// of TraditionalMAS32 and the 16-slot bank of CEMAS16.
//
// Integer work, bit-exact with the reference's definition
// (StiffGIPC/TraditionalMAS32Preconditioner.cu:463-1061, :1550-1962,
// :2142-2230; the same kernels with BANKSIZE 16 in
// StiffGIPC/MASPreconditioner.cu:29-628, :1132-1545, :1545-1818).  The
// reference runs one thread per slot and talks through shared memory; here
// kB consecutive lanes of a warp own one kB-slot bank (a whole warp for
// MAS32, half a warp for CEMAS16), the connected-component closure runs on
// shuffles of width kB, and every level count stays on the device (kernels
// read it) so the whole hierarchy is issued without a host round trip.
// Atomic ORs and integer atomic adds are order independent, so the results
// do not depend on scheduling.
#include "maspcg_internal.cuh"

namespace maspcg {
namespace {

constexpr int kTpb = 256;

__device__ __forceinline__ uint32_t lanemask_lt(int lane) { return (1u << lane) - 1u; }

// Ballot over the calling lane's bank: bit l for lane l of the bank.
template <int kB>
__device__ __forceinline__ uint32_t bank_ballot(bool p)
{
  const uint32_t b = __ballot_sync(kFull, p);
  if constexpr (kB == 32)
    return b;
  else
    return (b >> ((threadIdx.x & 31) & ~(kB - 1))) & ((1u << kB) - 1u);
}

// _buildCML0_new (:463-...): intra-bank neighbour bits, compact the rest.
template <int kB>
__global__ void k_cml0(const uint32_t* __restrict__ nstart, uint32_t* nnum, uint32_t* nlist, uint32_t* fine_mask,
                       const int* __restrict__ pmr, const int* __restrict__ rmp, int c0)
{
  const int tdx = blockIdx.x * blockDim.x + threadIdx.x;
  if (tdx >= c0) return;
  const int idx = pmr[tdx];
  if (idx < 0) return;
  const int bank = tdx / kB, lane = tdx % kB;
  uint32_t mask = 1u << lane;
  uint32_t nk = 0;
  const uint32_t st = nstart[idx], cnt = nnum[idx];
  for (uint32_t i = 0; i < cnt; ++i) {
    const uint32_t v = nlist[st + i];
    const int pv = rmp[v];
    if (pv / kB == bank)
      mask |= 1u << (uint32_t)(pv % kB);
    else
      nlist[st + nk++] = v;
  }
  nnum[idx] = nk;
  fine_mask[idx] = mask;
}

// int4 decoding of _buildCollisionConnection_new (:1550-1962).
__device__ __forceinline__ int decode_pair(int4 p, int* v)
{
  int x = p.x, y = p.y, z = p.z, w = p.w, cnt;
  if (x >= 0) {
    if (w < 0) w = -w - 1;
    cnt = 4;
  } else {
    x = -x - 1;
    if (z < 0) {
      if (y < 0) {
        y = -y - 1;
        z = -z - 1;
        w = -w - 1;
        cnt = 4;
      } else {
        cnt = 2;
      }
    } else if (w < 0) {
      if (y < 0) {
        y = -y - 1;
        w = -w - 1;
        cnt = 4;
      } else {
        cnt = 3;
      }
    } else {
      cnt = 4;
    }
  }
  v[0] = x;
  v[1] = y;
  v[2] = z;
  v[3] = w;
  return cnt;
}

// level < 0: fine level (masks indexed by vertex, ids are slots);
// level >= 1: masks indexed by the level's coarse node.
template <int kB>
__global__ void k_collision(uint32_t* connect, const int* __restrict__ cst_level, const int4* __restrict__ pairs,
                            const int* __restrict__ rmp, int node_offset, int nv, int n_pairs)
{
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_pairs) return;
  int v[4];
  const int cnt = decode_pair(pairs[p], v);
  int cp[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (i >= cnt) break;
    v[i] -= node_offset;
    if (v[i] >= nv) v[i] = -1;  // rejected on the host; defensive
    cp[i] = (v[i] >= 0) ? (cst_level ? cst_level[v[i]] : rmp[v[i]]) : -1;
  }
  uint32_t conn[4] = {0, 0, 0, 0};
  for (int i = 0; i < cnt; ++i)
    for (int j = i + 1; j < cnt; ++j) {
      const uint32_t my = (uint32_t)cp[i], ot = (uint32_t)cp[j];
      if (my == ot) continue;
      if (my / kB == ot / kB) {
        conn[i] |= 1u << (ot % kB);
        conn[j] |= 1u << (my % kB);
      }
    }
  for (int i = 0; i < cnt; ++i) {
    if (cst_level) {
      if (cp[i] >= 0) atomicOr(connect + cp[i], conn[i]);
    } else {
      if (v[i] >= 0) atomicOr(connect + v[i], conn[i]);
    }
  }
}

// Closure of the per-lane masks inside one bank: every lane walks the lanes
// reachable from it (the loop of _preparePrefixSumL0_new / _nextLevelCluster;
// both references stop early on an all-ones 32-bit mask, which a 16-slot
// mask never is).  The whole warp takes part; inactive lanes idle.
template <int kB>
__device__ __forceinline__ uint32_t bank_closure(bool active, uint32_t mask, uint32_t cache, int lane)
{
  uint32_t visited = 1u << lane;
  for (;;) {
    const uint32_t todo = (active && mask != kFull) ? (visited ^ mask) : 0u;
    const bool go = todo != 0u;
    if (!__any_sync(kFull, go)) break;
    const int nxt = go ? __ffs(todo) - 1 : lane;
    const uint32_t got = __shfl_sync(kFull, cache, nxt, kB);
    if (go) {
      visited |= 1u << nxt;
      mask |= got;
    }
  }
  return mask;
}

// _preparePrefixSumL0_new (:560-620).  Lanes of a bank past `banks` (the
// second half of the last warp when kB = 16) stay in the warp as inactive.
template <int kB>
__global__ void k_prefix_l0(uint32_t* fine_mask, int* prefix_orig, const int* __restrict__ pmr, int banks)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int bank = t / kB, lane = t % kB;
  if ((t & ~31) >= banks * kB) return;  // whole warp past the last bank
  const bool in = bank < banks;
  const int idx = in ? pmr[t] : -1;
  const bool real = idx >= 0;
  const uint32_t cache = real ? fine_mask[idx] : 0u;
  const uint32_t mask = bank_closure<kB>(real, cache, cache, lane);
  if (real) fine_mask[idx] = mask;
  const bool elected = real && __popc(mask & lanemask_lt(lane)) == 0;
  const int count = __popc(bank_ballot<kB>(elected));
  if (lane == 0 && real) prefix_orig[bank] = count;
}

// Exclusive scan of n ints (n read from *n_dev when n_dev != nullptr,
// else n_host), one CTA.  Also writes the total to *total when given.
template <typename T>
__global__ void k_scan_excl(const T* __restrict__ in, T* out, const int* n_dev, int n_host, int n_divisor)
{
  __shared__ T part[1024];
  int n = n_dev ? *n_dev : n_host;
  if (n_divisor > 1) n = (n + n_divisor - 1) / n_divisor;
  const int t = threadIdx.x;
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int lo = t * per, hi = min(lo + per, n);
  T s = 0;
  for (int i = lo; i < hi; ++i) s += in[i];
  part[t] = s;
  __syncthreads();
  // Hillis-Steele inclusive scan over the per-thread totals
  for (int o = 1; o < (int)blockDim.x; o <<= 1) {
    const T v = (t >= o) ? part[t - o] : T(0);
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  T acc = (t > 0) ? part[t - 1] : T(0);
  for (int i = lo; i < hi; ++i) {
    const T v = in[i];
    out[i] = acc;
    acc += v;
  }
}

// _buildLevel1_new (:681-744)
template <int kB>
__global__ void k_level1(int* level_size, int* cst, int* going_next, const uint32_t* __restrict__ fine_mask,
                         const int* __restrict__ prefix_sum, const int* __restrict__ prefix_orig,
                         const int* __restrict__ pmr, int c0)
{
  const int tdx = blockIdx.x * blockDim.x + threadIdx.x;
  const int bank = tdx / kB, lane = tdx % kB;
  const int banks = c0 / kB;
  if ((tdx & ~31) >= banks * kB) return;
  const bool in = bank < banks;
  const int padded = (c0 + kB - 1) / kB * kB;
  if (tdx == c0 - 1) {
    level_size[2] = prefix_sum[bank] + prefix_orig[bank];
    level_size[3] = padded;
  }
  const int idx = in ? pmr[tdx] : -1;
  const bool real = idx >= 0;
  const uint32_t mask = real ? fine_mask[idx] : 0u;
  const bool elected = real && __popc(mask & lanemask_lt(lane)) == 0;
  const uint32_t em = bank_ballot<kB>(elected);
  const int lane_prefix = __popc(em & lanemask_lt(lane)) + (in ? prefix_sum[bank] : 0);
  const int el = real ? __ffs(mask) - 1 : lane;
  const int coarse = __shfl_sync(kFull, lane_prefix, el, kB);
  if (real) {
    cst[idx] = coarse;
    going_next[idx] = coarse + padded;
  }
}

// _buildConnectMaskLx_new (:821-903)
template <int kB>
__global__ void k_connect_lx(const uint32_t* __restrict__ nstart, uint32_t* nnum, uint32_t* nlist,
                             const int* __restrict__ cst_prev, uint32_t* next_mask, const uint32_t* __restrict__ fine_mask,
                             const int* __restrict__ pmr, int banks)
{
  __shared__ uint32_t cache_s[kTpb];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int bank = t / kB, lane = t % kB;
  if ((t & ~31) >= banks * kB) return;
  uint32_t* cache = cache_s + (threadIdx.x / kB) * kB;
  const int idx = bank < banks ? pmr[t] : -1;
  const bool real = idx >= 0;
  uint32_t prefix = 0, conn = 0, coarse = 0;
  if (real) {
    prefix = fine_mask[idx];
    coarse = (uint32_t)cst_prev[idx];
    uint32_t nk = 0;
    const uint32_t st = nstart[idx], cnt = nnum[idx];
    for (uint32_t i = 0; i < cnt; ++i) {
      const uint32_t u = nlist[st + i];
      const uint32_t cc = (uint32_t)cst_prev[u];
      if (coarse / kB == cc / kB)
        conn |= 1u << (cc % kB);
      else
        nlist[st + nk++] = u;
    }
    nnum[idx] = nk;
    cache[lane] = 0u;
  }
  __syncwarp();
  int ci = 0;
  if (real) {
    if (__popc(prefix) == kB) {
      atomicOr(cache, conn);
      ci = 0;
    } else {
      const int e = __ffs(prefix) - 1;
      if (conn) atomicOr(cache + e, conn);
      ci = e;
    }
  }
  __syncwarp();
  if (real) {
    const uint32_t cm = cache[ci];
    if (cm && __popc(prefix & lanemask_lt(lane)) == 0) atomicOr(next_mask + coarse, cm);
  }
}

// _nextLevelCluster (:905-956); the level's node count is read on the device.
template <int kB>
__global__ void k_next_cluster(uint32_t* next_mask, uint32_t* next_prefix, const int* __restrict__ level_size,
                               int level, int max_banks)
{
  const int number = level_size[2 * level];
  const int banks = min((number + kB - 1) / kB, max_banks);
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int bank = idx / kB, lane = idx % kB;
  if ((idx & ~31) >= banks * kB) return;
  const bool valid = bank < banks && idx < number;
  const uint32_t cache = valid ? ((1u << lane) | next_mask[idx]) : 0u;
  const uint32_t mask = bank_closure<kB>(valid, cache, cache, lane);
  if (valid) next_mask[idx] = mask;
  const bool elected = valid && __popc(mask & lanemask_lt(lane)) == 0;
  const int count = __popc(bank_ballot<kB>(elected));
  if (lane == 0 && bank < banks) next_prefix[bank] = (uint32_t)count;
}

// _prefixSumLx (:958-1009)
template <int kB>
__global__ void k_prefix_lx(int* level_size, const uint32_t* __restrict__ next_prefix,
                            const uint32_t* __restrict__ next_prefix_sum, uint32_t* next_mask, int* going_next,
                            int level, int max_banks)
{
  const int number = level_size[2 * level];
  const int begin = level_size[2 * level + 1];
  const int banks = min((number + kB - 1) / kB, max_banks);
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int bank = idx / kB, lane = idx % kB;
  if ((idx & ~31) >= banks * kB) return;
  const bool in = bank < banks;
  const bool valid = in && idx < number;
  const int padded = (number + kB - 1) / kB * kB;
  if (in && idx == number - 1) {
    level_size[2 * (level + 1)] = (int)(next_prefix_sum[bank] + next_prefix[bank]);
    level_size[2 * (level + 1) + 1] = begin + padded;
  }
  const uint32_t mask = valid ? next_mask[idx] : 0u;
  const bool elected = valid && __popc(mask & lanemask_lt(lane)) == 0;
  const uint32_t em = bank_ballot<kB>(elected);
  const int lane_prefix = __popc(em & lanemask_lt(lane)) + (in ? (int)next_prefix_sum[bank] : 0);
  const int el = valid ? __ffs(mask) - 1 : lane;
  const int coarse = __shfl_sync(kFull, lane_prefix, el, kB);
  if (valid) {
    next_mask[idx] = (uint32_t)coarse;
    going_next[idx + begin] = coarse + begin + padded;
  }
}

// _computeNextLevel (:1011-1022)
__global__ void k_compute_next(int* cst, const uint32_t* __restrict__ next_mask, int level, int nv)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nv) return;
  const int next = cst[(size_t)(level - 1) * nv + idx];
  cst[(size_t)level * nv + idx] = (int)next_mask[next];
}

// _aggregationKernel (:1024-1058): chain of coarse slots per vertex.
__global__ void k_aggregate(int* coarse_table, const int* __restrict__ going_next, int levelnum, int nv)
{
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nv) return;
  int cur = idx;
  int t[6] = {-1, -1, -1, -1, -1, -1};
  for (int l = 0; l < levelnum - 1; ++l) {
    cur = going_next[cur];
    t[l] = cur;
  }
#pragma unroll
  for (int l = 0; l < 6; ++l) coarse_table[(size_t)idx * 6 + l] = t[l];
}

// Level-L node of every fine slot (-1 for padding slots): the keys of the
// member lists used by the domain assembly and the restriction.
__global__ void k_slot_map(int* cmap, const int* __restrict__ cst_level, const int* __restrict__ pmr, int c0)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= c0) return;
  const int v = pmr[s];
  cmap[s] = v >= 0 ? cst_level[v] : -1;
}

template <int kB>
void build_hierarchy_t(maspcg_handle* h)
{
  cudaStream_t st = h->stream;
  const int nv = h->nv, c0 = h->c0, L = h->levelnum;
  const int banks0 = c0 / kB;
  // restore the compacted neighbour lists (setPreconditioner_bcoo :2643-2660)
  if (h->nlist_size > 0)
    MCK(cudaMemcpyAsync(h->nlist.get(), h->nlist_init.get(), (size_t)h->nlist_size * 4, cudaMemcpyDeviceToDevice, st));
  MCK(cudaMemcpyAsync(h->nnum.get(), h->nnum_init.get(), (size_t)nv * 4, cudaMemcpyDeviceToDevice, st));
  MCK(cudaMemsetAsync(h->level_size.get(), 0, sizeof(int) * 2 * (L + 1), st));
  MCK(cudaMemsetAsync(h->fine_mask.get(), 0, (size_t)nv * 4, st));

  const int4* pairs = reinterpret_cast<const int4*>(h->pairs.get());
  k_cml0<kB><<<ceil_div(c0, kTpb), kTpb, 0, st>>>(h->nstart.get(), h->nnum.get(), h->nlist.get(), h->fine_mask.get(),
                                             h->pmr.get(), h->rmp.get(), c0); MLAUNCHED(h);
  if (h->n_pairs) {
    k_collision<kB><<<ceil_div(h->n_pairs, kTpb), kTpb, 0, st>>>(h->fine_mask.get(), nullptr, pairs, h->rmp.get(),
                                                            h->node_offset, nv, h->n_pairs);
    MLAUNCHED(h);
  }
  k_prefix_l0<kB><<<ceil_div((long long)banks0 * kB, kTpb), kTpb, 0, st>>>(h->fine_mask.get(), h->prefix_orig.get(),
                                                                       h->pmr.get(), banks0); MLAUNCHED(h);
  k_scan_excl<int><<<1, 1024, 0, st>>>(h->prefix_orig.get(), h->prefix_sum_orig.get(), nullptr, banks0, 1); MLAUNCHED(h);
  k_level1<kB><<<ceil_div((long long)banks0 * kB, kTpb), kTpb, 0, st>>>(h->level_size.get(), h->cst.get(),
                                                                    h->going_next.get(), h->fine_mask.get(),
                                                                    h->prefix_sum_orig.get(), h->prefix_orig.get(),
                                                                    h->pmr.get(), c0); MLAUNCHED(h);
  const int max_banks = ceil_div(nv, kB);
  for (int level = 1; level < L; ++level) {
    MCK(cudaMemsetAsync(h->next_mask.get(), 0, (size_t)nv * 4, st));
    const int* cst_prev = h->cst.get() + (size_t)(level - 1) * nv;
    k_connect_lx<kB><<<ceil_div((long long)banks0 * kB, kTpb), kTpb, 0, st>>>(
        h->nstart.get(), h->nnum.get(), h->nlist.get(), cst_prev, h->next_mask.get(), h->fine_mask.get(),
        h->pmr.get(), banks0); MLAUNCHED(h);
    if (h->n_pairs) {
      k_collision<kB><<<ceil_div(h->n_pairs, kTpb), kTpb, 0, st>>>(h->next_mask.get(), cst_prev, pairs, h->rmp.get(),
                                                              h->node_offset, nv, h->n_pairs);
      MLAUNCHED(h);
    }
    k_next_cluster<kB><<<ceil_div((long long)max_banks * kB, kTpb), kTpb, 0, st>>>(
        h->next_mask.get(), h->next_prefix.get(), h->level_size.get(), level, max_banks); MLAUNCHED(h);
    k_scan_excl<uint32_t><<<1, 1024, 0, st>>>(h->next_prefix.get(), h->next_prefix_sum.get(),
                                              h->level_size.get() + 2 * level, 0, kB); MLAUNCHED(h);
    k_prefix_lx<kB><<<ceil_div((long long)max_banks * kB, kTpb), kTpb, 0, st>>>(
        h->level_size.get(), h->next_prefix.get(), h->next_prefix_sum.get(), h->next_mask.get(),
        h->going_next.get(), level, max_banks); MLAUNCHED(h);
    k_compute_next<<<ceil_div(nv, kTpb), kTpb, 0, st>>>(h->cst.get(), h->next_mask.get(), level, nv); MLAUNCHED(h);
  }
  k_aggregate<<<ceil_div(nv, kTpb), kTpb, 0, st>>>(h->coarse_table.get(), h->going_next.get(), L, nv); MLAUNCHED(h);
  MCK(cudaGetLastError());

  // One host read per build: the level sizes decide the domain count.
  std::vector<int> ls(2 * (L + 1));
  MCK(cudaMemcpyAsync(ls.data(), h->level_size.get(), sizeof(int) * ls.size(), cudaMemcpyDeviceToHost, st));
  MCK(cudaStreamSynchronize(st));
  LevelInfo lv{};
  lv.levelnum = L;
  lv.count[0] = c0;
  lv.begin[0] = 0;
  for (int l = 1; l <= L; ++l) {
    lv.count[l] = ls[2 * l];
    lv.begin[l] = ls[2 * l + 1];
  }
  lv.total_clusters = lv.begin[L];
  MREQ(lv.total_clusters > 0 && lv.total_clusters % kB == 0, MASPCG_ERR_CAPACITY, "invalid MAS level sizes");
  MREQ((long long)lv.total_clusters <= h->gn_cap, MASPCG_ERR_CAPACITY, "MAS hierarchy exceeds its capacity");
  for (int l = 0; l <= L; ++l) lv.dom_begin[l] = lv.begin[l] / kB;
  lv.domains = lv.total_clusters / kB;
  h->lv = lv;

  // level-L node of each fine slot
  for (int l = 1; l < L; ++l) {
    h->cmap[l].resize(c0);
    k_slot_map<<<ceil_div(c0, kTpb), kTpb, 0, st>>>(h->cmap[l].get(), h->cst.get() + (size_t)(l - 1) * nv,
                                                   h->pmr.get(), c0); MLAUNCHED(h);
  }
  MCK(cudaGetLastError());
}

}  // namespace

void build_hierarchy(maspcg_handle* h)
{
  if (h->bank == 16)
    build_hierarchy_t<16>(h);
  else
    build_hierarchy_t<32>(h);
}

}  // namespace maspcg
