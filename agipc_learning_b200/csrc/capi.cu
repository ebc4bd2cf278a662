// capi.cu -- the extern "C" boundary declared in include/maspcg.h.
//
// Every entry point validates its arguments, turns exceptions into a
// maspcg_status and keeps the message for maspcg_last_error; nothing aborts.
#include <algorithm>
#include <cmath>
#include <limits>
#include <new>
#include <vector>

#include "maspcg_internal.cuh"

using maspcg::DBuf;
using maspcg::Error;

namespace {

thread_local std::string g_create_error;

// The device of the handle the current entry point serves (set by guard), so
// a device pointer can be checked against it.
thread_local int g_call_device = -1;

// True for memory a kernel on the handle's device can read: managed memory,
// or device memory of that device.  Device memory of another GPU is refused
// (MASPCG_ERR_INVALID_ARGUMENT): without peer access a kernel given it would
// fault.
bool is_device_ptr(const void* p)
{
  if (!p) return false;
  cudaPointerAttributes at{};
  const cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (at.type == cudaMemoryTypeManaged) return true;
  if (at.type != cudaMemoryTypeDevice) return false;
  MREQ(g_call_device < 0 || at.device == g_call_device, MASPCG_ERR_INVALID_ARGUMENT,
       "device pointer on GPU " + std::to_string(at.device) + ", handle on GPU " + std::to_string(g_call_device));
  return true;
}

// A device view of a caller array: the caller's pointer when it is device
// memory, else a staged copy.
template <typename T>
const T* device_in(maspcg_handle* h, const T* user, size_t count, DBuf<T>& stage)
{
  if (count == 0) return nullptr;
  MREQ(user != nullptr, MASPCG_ERR_INVALID_ARGUMENT, "null array argument");
  if (is_device_ptr(user)) return user;
  stage.resize(count);
  MCK(cudaMemcpyAsync(stage.get(), user, count * sizeof(T), cudaMemcpyHostToDevice, h->stream));
  return stage.get();
}

template <typename T>
std::vector<T> host_copy(maspcg_handle* h, const T* user, size_t count)
{
  std::vector<T> v(count);
  if (!count) return v;
  MREQ(user != nullptr, MASPCG_ERR_INVALID_ARGUMENT, "null array argument");
  if (is_device_ptr(user)) {
    MCK(cudaMemcpyAsync(v.data(), user, count * sizeof(T), cudaMemcpyDeviceToHost, h->stream));
    MCK(cudaStreamSynchronize(h->stream));
  } else {
    std::copy(user, user + count, v.begin());
  }
  return v;
}

// Runs one entry point on the handle's device and puts the caller's current
// device back afterwards, on every path: the reference runs on the caller's
// device and never changes it.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int device)
  {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
    }
    if (prev != device) MCK(cudaSetDevice(device));
    g_call_device = device;
  }
  ~DeviceScope()
  {
    g_call_device = -1;
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

template <typename F>
maspcg_status guard(maspcg_handle* h, F&& f)
{
  if (!h) return MASPCG_ERR_NULL_HANDLE;
  try {
    DeviceScope scope(h->device);
    f();
    h->last_error.clear();
    return MASPCG_OK;
  } catch (const Error& e) {
    h->last_error = e.what();
    return e.status;
  } catch (const std::bad_alloc&) {
    h->last_error = "host allocation failed";
    return MASPCG_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    h->last_error = e.what();
    return MASPCG_ERR_CUDA;
  }
}

int compute_num_levels(int vert_num, int bank)
{
  // computeNumLevels (TraditionalMAS32Preconditioner.cu:2142-2161,
  // MASPreconditioner.cu:1727-1746 with BANKSIZE 16)
  int n_level = 1;
  int level_sz = (vert_num + bank - 1) / bank * bank;
  while (level_sz > bank) {
    level_sz /= bank;
    n_level++;
    level_sz = (level_sz + bank - 1) / bank * bank;
  }
  n_level += 1;
  return n_level > 6 ? 6 : n_level;
}

long long hierarchy_capacity(long long vertices, long long mapped, long long levels, long long bank)
{
  // gipc::hierarchy_capacity (gipc/hierarchy_capacity.h:10-22)
  const long long base = std::max(vertices, mapped);
  if (!base || !levels) return 0;
  const long long maximum = (long long)(((unsigned long long)-1 >> 1) / sizeof(unsigned int));
  MREQ(bank && base <= maximum && bank - 1 <= maximum - base, MASPCG_ERR_CAPACITY, "MAS hierarchy alignment overflow");
  const long long padded = (base + bank - 1) / bank * bank;
  MREQ(padded <= maximum / levels, MASPCG_ERR_CAPACITY, "MAS hierarchy capacity overflow");
  MREQ(padded * levels <= 0x7fffffffLL, MASPCG_ERR_CAPACITY, "MAS hierarchy exceeds 32-bit indices");
  return padded * levels;
}

void alloc_vectors(maspcg_handle* h)
{
  const size_t n = 3 * (size_t)h->nb_int;
  const size_t es = maspcg::vec_elem_size(h);
  for (auto* b : {&h->vx, &h->vr, &h->vz, &h->vap}) b->resize(n * es);
  h->vp4.resize(4 * (size_t)h->nb_int * es, 32);
  h->b64.resize(n);
  h->x64.resize(n);
  h->r64.resize(n);
  const size_t io = 3 * (size_t)std::max(h->nb, h->nb_int);
  h->io_a.resize(io);
  h->io_b.resize(io);
  const int parts = 32 * h->sm_count + 64;
  h->partial.resize(parts);
  h->partial_rz.resize(parts);
  h->partial_rr.resize(parts);
  if (h->cfg.precision != MASPCG_PREC_REFERENCE) h->vr2.resize(n * 4);
}

}  // namespace

namespace {
// A device output array, or handle scratch copied back to the host one.
template <typename T>
T* device_out(T* user, size_t count, maspcg::DBuf<T>& stage)
{
  if (is_device_ptr(user)) return user;
  stage.resize(std::max<size_t>(count, 1));
  return stage.get();
}
template <typename T>
void copy_back(maspcg_handle* h, T* user, const T* dev, size_t count)
{
  if (count && dev != user)
    MCK(cudaMemcpyAsync(user, dev, count * sizeof(T), cudaMemcpyDeviceToHost, h->stream));
}
}  // namespace

namespace {
// Validate a coarse mapping on host copies and stage its arrays on the device.
maspcg::GalerkinMap galerkin_map(maspcg_handle* h, const maspcg_galerkin_map* map)
{
  MREQ(map != nullptr, MASPCG_ERR_INVALID_ARGUMENT, "null mapping");
  const maspcg_galerkin_map& g = *map;
  MREQ(g.prefix_blocks >= 0 && g.fem_nodes >= 0 && g.coarse_nodes >= 0 && g.coarse_block_nodes >= 0,
       MASPCG_ERR_INVALID_ARGUMENT, "negative mapping size");
  MREQ(g.fem_nodes == 0 || g.coarse_nodes > 0, MASPCG_ERR_INVALID_ARGUMENT, "mapping has no coarse owner");
  MREQ((long long)g.prefix_blocks + g.fem_nodes <= 0x7fffffffLL &&
           (long long)g.prefix_blocks + g.coarse_block_nodes <= 0x7fffffffLL,
       MASPCG_ERR_CAPACITY, "block count overflow");
  if (g.fem_nodes > 0) {
    const std::vector<int> f2c = host_copy(h, g.fine_to_coarse, (size_t)g.fem_nodes);
    const std::vector<int> base = host_copy(h, g.coarse_block_bases, (size_t)g.coarse_nodes);
    const std::vector<int> mask = host_copy(h, g.basis_masks, (size_t)g.coarse_nodes);
    for (int c : f2c) MREQ(c >= 0 && c < g.coarse_nodes, MASPCG_ERR_INVALID_ARGUMENT, "fine_to_coarse out of range");
    for (int c = 0; c < g.coarse_nodes; ++c) {
      MREQ(mask[c] >= 1 && mask[c] <= 15, MASPCG_ERR_INVALID_ARGUMENT, "basis mask outside 1..15");
      int w = 0;
      for (int q = 0; q < 4; ++q) w += (mask[c] >> q) & 1;
      MREQ(base[c] >= 0 && (long long)base[c] + w <= g.coarse_block_nodes, MASPCG_ERR_INVALID_ARGUMENT,
           "coarse block base out of range");
    }
  }
  maspcg::GalerkinMap m{};
  m.prefix = g.prefix_blocks;
  m.fine_blocks = g.prefix_blocks + g.fem_nodes;
  if (g.fem_nodes > 0) {
    m.fine_to_coarse = device_in(h, g.fine_to_coarse, (size_t)g.fem_nodes, h->gal_f2c);
    m.coarse_block_bases = device_in(h, g.coarse_block_bases, (size_t)g.coarse_nodes, h->gal_bases);
    m.basis_masks = device_in(h, g.basis_masks, (size_t)g.coarse_nodes, h->gal_masks);
    m.rest = device_in(h, g.rest_positions, 3 * (size_t)g.fem_nodes, h->gal_rest);
  }
  return m;
}
}  // namespace

namespace {
// In-place triplet fix-up shared by the two entry points below: stage host
// arrays, run the kernel, copy them back.
maspcg_status triplet_fixup(maspcg_handle* h, int n, int* rows, int* cols, double* values9, const int* bd_type,
                            int n_vertices, int offset, bool zero_boundary_only)
{
  return guard(h, [&] {
    MREQ(n >= 0 && n_vertices >= 0, MASPCG_ERR_INVALID_ARGUMENT, "negative count");
    if (n == 0) return;
    MREQ(rows && cols && values9 && bd_type, MASPCG_ERR_INVALID_ARGUMENT, "null array argument");
    MREQ(n_vertices > 0, MASPCG_ERR_INVALID_ARGUMENT, "no vertices");
    const bool dev_rows = is_device_ptr(rows), dev_cols = is_device_ptr(cols), dev_vals = is_device_ptr(values9);
    int* r = dev_rows ? rows : const_cast<int*>(device_in(h, (const int*)rows, (size_t)n, h->asm_rows));
    int* c = dev_cols ? cols : const_cast<int*>(device_in(h, (const int*)cols, (size_t)n, h->asm_cols));
    double* v = dev_vals ? values9 : const_cast<double*>(device_in(h, (const double*)values9, 9 * (size_t)n, h->asm_vals));
    const int* bd = device_in(h, bd_type, (size_t)n_vertices, h->asm_start);
    const bool ok = maspcg::adjust_contacts(h, n, r, c, v, bd, n_vertices, offset, zero_boundary_only);
    if (!zero_boundary_only && !dev_rows) copy_back(h, rows, (const int*)r, (size_t)n);
    if (!zero_boundary_only && !dev_cols) copy_back(h, cols, (const int*)c, (size_t)n);
    if (!dev_vals) copy_back(h, values9, (const double*)v, 9 * (size_t)n);
    MCK(cudaStreamSynchronize(h->stream));
    MREQ(ok, MASPCG_ERR_INVALID_ARGUMENT, "a triplet names a vertex outside [0, n_vertices); it was left unchanged");
  });
}
}  // namespace

extern "C" {

MASPCG_API void maspcg_config_default(maspcg_config* c)
{
  if (!c) return;
  c->tolerance = 1e-4;
  c->max_iter_ratio = 0.3;
  c->max_iterations = 0;
  c->gate = MASPCG_GATE_RZ;
  c->precision = MASPCG_PREC_REFERENCE;
  c->inverse_storage = MASPCG_INV_FP32;
  c->preconditioner = MASPCG_PRECOND_MAS32;
  c->refinement_period = 16;
  c->bank_size = 32;
  c->iterations_per_launch = 8;
  c->flags = 0;
  c->matrix_form = MASPCG_MATRIX_F32;
  c->residual_replacement = MASPCG_REPLACE_PERIODIC;
}

MASPCG_API const char* maspcg_status_string(int s)
{
  switch (s) {
    case MASPCG_OK: return "ok";
    case MASPCG_ERR_INVALID_ARGUMENT: return "invalid argument";
    case MASPCG_ERR_NULL_HANDLE: return "null handle";
    case MASPCG_ERR_CUDA: return "CUDA error";
    case MASPCG_ERR_OUT_OF_MEMORY: return "out of memory";
    case MASPCG_ERR_NOT_READY: return "not ready (call order)";
    case MASPCG_ERR_CAPACITY: return "capacity exceeded";
    case MASPCG_ERR_NO_DEVICE: return "no CUDA device";
    case MASPCG_ERR_UNSUPPORTED: return "unsupported configuration";
    default: return "unknown status";
  }
}

MASPCG_API const char* maspcg_last_error(const maspcg_handle* h)
{
  return h ? h->last_error.c_str() : g_create_error.c_str();
}

MASPCG_API maspcg_status maspcg_create(const maspcg_config* cfg, maspcg_handle** out)
{
  g_create_error.clear();
  if (!out) {
    g_create_error = "out is null";
    return MASPCG_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  maspcg_config c;
  maspcg_config_default(&c);
  if (cfg) c = *cfg;
  if (c.bank_size != 32 && c.bank_size != 16) {
    g_create_error = "the MAS bank is 32 (TraditionalMAS32) or 16 (CEMAS16) vertices";
    return MASPCG_ERR_UNSUPPORTED;
  }
  if ((c.preconditioner == MASPCG_PRECOND_MAS32 && c.bank_size != 32) ||
      (c.preconditioner == MASPCG_PRECOND_MAS16 && c.bank_size != 16)) {
    g_create_error = "MAS32 takes the 32-vertex bank, CEMAS16 the 16-vertex bank";
    return MASPCG_ERR_UNSUPPORTED;
  }
  if (c.preconditioner == MASPCG_PRECOND_MAS16 && c.inverse_storage != MASPCG_INV_FP32) {
    g_create_error = "CEMAS16 stores FP32 inverses";
    return MASPCG_ERR_UNSUPPORTED;
  }
  if (!(c.tolerance > 0) || c.precision < 0 || c.precision > 2 || c.gate < 0 || c.gate > 1 ||
      c.inverse_storage < 0 || c.inverse_storage > 2 ||
      !(c.preconditioner == MASPCG_PRECOND_BLOCK_JACOBI || c.preconditioner == MASPCG_PRECOND_MAS32 ||
        c.preconditioner == MASPCG_PRECOND_MAS16 || c.preconditioner == MASPCG_PRECOND_NONE) ||
      c.max_iterations < 0 || !(c.max_iter_ratio >= 0) || (c.flags & ~127) != 0 || c.matrix_form < 0 ||
      c.matrix_form > 3 || c.residual_replacement < 0 || c.residual_replacement > 1 ||
      ((c.flags & MASPCG_FLAG_APPLY_STAGED2) && (c.flags & MASPCG_FLAG_APPLY_DIRECT))) {
    g_create_error = "invalid configuration";
    return MASPCG_ERR_INVALID_ARGUMENT;
  }
  if (c.refinement_period <= 0) c.refinement_period = 16;
  if (c.iterations_per_launch <= 0) c.iterations_per_launch = 8;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    g_create_error = "no CUDA device";
    return MASPCG_ERR_NO_DEVICE;
  }
  maspcg_handle* h = nullptr;
  try {
    h = new maspcg_handle();
    h->cfg = c;
    MCK(cudaGetDevice(&h->device));
    MCK(cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, h->device));
    MCK(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    h->stream = h->own_stream;
    MCK(cudaEventCreate(&h->ev0));
    MCK(cudaEventCreate(&h->ev1));
    MCK(cudaMallocHost(reinterpret_cast<void**>(&h->h_scal), sizeof(maspcg::PcgScalars)));
    MCK(cudaMallocHost(reinterpret_cast<void**>(&h->h_err), sizeof(int)));
    h->scal.resize(1);
    h->grid_stream = 4 * h->sm_count;
    h->use_pdl = (c.flags & MASPCG_FLAG_PDL) != 0;
    // reference precision keeps the reference's r.z: summed over the fine
    // rows after the coarse correction is added to z
    h->overlap_coarse = (c.flags & MASPCG_FLAG_SEQUENTIAL_COARSE) == 0 && c.precision != MASPCG_PREC_REFERENCE;
    h->fused_head = (c.flags & MASPCG_FLAG_FUSED_HEAD) != 0;
    h->fuse_update = (c.flags & MASPCG_FLAG_FUSED_UPDATE) != 0;
    MCK(cudaStreamCreateWithFlags(&h->side_stream, cudaStreamNonBlocking));
    MCK(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
    MCK(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
    h->apply_variant = (c.flags & MASPCG_FLAG_APPLY_STAGED2) ? 1 : (c.flags & MASPCG_FLAG_APPLY_DIRECT) ? 0 : 2;
    h->failed.resize(8);
    MCK(cudaMemset(h->failed.get(), 0, 8 * sizeof(int)));
  } catch (const std::exception& e) {
    g_create_error = e.what();
    if (h) maspcg_destroy(h);
    return MASPCG_ERR_CUDA;
  }
  *out = h;
  return MASPCG_OK;
}

MASPCG_API maspcg_status maspcg_destroy(maspcg_handle* h)
{
  if (!h) return MASPCG_ERR_NULL_HANDLE;
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->side_stream) cudaStreamSynchronize(h->side_stream);
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  if (h->h_scal) cudaFreeHost(h->h_scal);
  if (h->h_err) cudaFreeHost(h->h_err);
  if (h->side_stream) cudaStreamDestroy(h->side_stream);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
  return MASPCG_OK;
}

MASPCG_API maspcg_status maspcg_set_stream(maspcg_handle* h, void* stream)
{
  return guard(h, [&] {
    MCK(cudaStreamSynchronize(h->stream));
    h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own_stream;
    h->graph_dirty = true;
  });
}

MASPCG_API maspcg_status maspcg_get_stream(const maspcg_handle* h, void** stream)
{
  if (!h || !stream) return MASPCG_ERR_INVALID_ARGUMENT;
  *stream = static_cast<void*>(h->stream);
  return MASPCG_OK;
}

MASPCG_API maspcg_status maspcg_set_graph(maspcg_handle* h, int vert_num, int collision_node_offset,
                                          const uint32_t* neighbor_start, const uint32_t* neighbor_num,
                                          const uint32_t* neighbor_list, int neighbor_list_size,
                                          const int* part_map_real, int part_map_size, const int* real_map_part)
{
  return guard(h, [&] {
    const int bank = h->cfg.bank_size;
    MREQ(vert_num >= 1, MASPCG_ERR_INVALID_ARGUMENT, "vert_num must be >= 1");
    MREQ(part_map_size >= vert_num && part_map_size % bank == 0, MASPCG_ERR_INVALID_ARGUMENT,
         bank == 16 ? "part_map_size must be a multiple of 16 and >= vert_num"
                    : "part_map_size must be a multiple of 32 and >= vert_num");
    MREQ(neighbor_list_size >= 0, MASPCG_ERR_INVALID_ARGUMENT, "negative neighbor_list_size");
    const auto st = host_copy(h, neighbor_start, vert_num);
    const auto nn = host_copy(h, neighbor_num, vert_num);
    const auto nl = host_copy(h, neighbor_list, (size_t)neighbor_list_size);
    const auto pmr = host_copy(h, part_map_real, part_map_size);
    const auto rmp = host_copy(h, real_map_part, vert_num);
    for (int v = 0; v < vert_num; ++v) {
      MREQ((long long)st[v] + nn[v] <= neighbor_list_size, MASPCG_ERR_INVALID_ARGUMENT,
           "neighbour range exceeds the list");
      MREQ(rmp[v] >= 0 && rmp[v] < part_map_size, MASPCG_ERR_INVALID_ARGUMENT, "real_map_part out of range");
      MREQ(pmr[rmp[v]] == v, MASPCG_ERR_INVALID_ARGUMENT, "part_map_real / real_map_part disagree");
    }
    for (int i = 0; i < neighbor_list_size; ++i)
      MREQ(nl[i] < (uint32_t)vert_num, MASPCG_ERR_INVALID_ARGUMENT, "neighbour index out of range");
    int mapped = 0;
    for (int s = 0; s < part_map_size; ++s) {
      MREQ(pmr[s] >= -1 && pmr[s] < vert_num, MASPCG_ERR_INVALID_ARGUMENT, "part_map_real out of range");
      mapped += pmr[s] >= 0;
    }
    MREQ(mapped == vert_num, MASPCG_ERR_INVALID_ARGUMENT, "part_map_real must map every vertex once");
    for (int b = 0; b < part_map_size / bank; ++b)
      MREQ(pmr[bank * b] >= 0, MASPCG_ERR_INVALID_ARGUMENT,
           bank == 16 ? "lane 0 of every 16-slot bank must hold a vertex"
                      : "lane 0 of every 32-slot bank must hold a vertex");

    h->bank = bank;
    h->nv = vert_num;
    h->c0 = part_map_size;
    h->node_offset = collision_node_offset;
    h->nlist_size = neighbor_list_size;
    h->levelnum = compute_num_levels(std::max(part_map_size, vert_num), bank);
    h->gn_cap = hierarchy_capacity(vert_num, part_map_size, h->levelnum, bank);
    cudaStream_t s = h->stream;
    auto up = [&](auto& buf, const auto& vec) {
      buf.resize(std::max<size_t>(vec.size(), 1));
      if (!vec.empty())
        MCK(cudaMemcpyAsync(buf.get(), vec.data(), vec.size() * sizeof(vec[0]), cudaMemcpyHostToDevice, s));
    };
    up(h->nstart, st);
    up(h->nnum_init, nn);
    up(h->nlist_init, nl);
    h->nnum.resize(vert_num);
    h->nlist.resize(std::max(neighbor_list_size, 1));
    up(h->pmr, pmr);
    up(h->rmp, rmp);
    h->h_pmr = pmr;
    h->h_rmp = rmp;
    const int L = h->levelnum;
    h->fine_mask.resize(vert_num);
    h->next_mask.resize(vert_num);
    h->next_prefix.resize(vert_num / bank + 2);
    h->next_prefix_sum.resize(vert_num / bank + 2);
    h->prefix_orig.resize(part_map_size / bank + 1);
    h->prefix_sum_orig.resize(part_map_size / bank + 1);
    h->cst.resize((size_t)vert_num * L);
    h->going_next.resize((size_t)h->gn_cap);
    MCK(cudaMemsetAsync(h->going_next.get(), 0xff, (size_t)h->gn_cap * 4, s));
    h->coarse_table.resize((size_t)vert_num * 6);
    h->level_size.resize(2 * (L + 1));
    MCK(cudaStreamSynchronize(s));
    h->has_graph = true;
    h->has_matrix = h->has_precond = false;
    h->graph_dirty = true;
  });
}

MASPCG_API maspcg_status maspcg_set_contacts(maspcg_handle* h, const int* pairs4, int n_pairs)
{
  return guard(h, [&] {
    MREQ(h->has_graph, MASPCG_ERR_NOT_READY, "set_graph first");
    MREQ(n_pairs >= 0, MASPCG_ERR_INVALID_ARGUMENT, "negative pair count");
    const auto p = host_copy(h, pairs4, 4 * (size_t)n_pairs);
    for (int i = 0; i < n_pairs; ++i) {
      int x = p[4 * i], y = p[4 * i + 1], z = p[4 * i + 2], w = p[4 * i + 3];
      int v[4], cnt;
      // decoding of _buildCollisionConnection_new (:1550-1962)
      if (x >= 0) {
        if (w < 0) w = -w - 1;
        cnt = 4;
      } else {
        x = -x - 1;
        if (z < 0) {
          if (y < 0) { y = -y - 1; z = -z - 1; w = -w - 1; cnt = 4; }
          else cnt = 2;
        } else if (w < 0) {
          if (y < 0) { y = -y - 1; w = -w - 1; cnt = 4; }
          else cnt = 3;
        } else cnt = 4;
      }
      v[0] = x; v[1] = y; v[2] = z; v[3] = w;
      for (int q = 0; q < cnt; ++q)
        MREQ(v[q] - h->node_offset < h->nv, MASPCG_ERR_INVALID_ARGUMENT, "contact vertex beyond the FEM range");
    }
    h->pairs.resize(std::max<size_t>(4 * (size_t)n_pairs, 4));
    if (n_pairs)
      MCK(cudaMemcpyAsync(h->pairs.get(), p.data(), p.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    MCK(cudaStreamSynchronize(h->stream));
    h->n_pairs = n_pairs;
    h->has_precond = false;
  });
}

namespace {
void check_matrix_args(maspcg_handle* h, int n_blocks, int block_rows, int fem_offset_blocks, int abd_body_count)
{
  MREQ(n_blocks >= 1 && block_rows >= 1, MASPCG_ERR_INVALID_ARGUMENT, "empty matrix");
  MREQ(fem_offset_blocks >= 0 && abd_body_count >= 0 && 4LL * abd_body_count <= block_rows,
       MASPCG_ERR_INVALID_ARGUMENT, "invalid offsets");
  MREQ(n_blocks <= (1 << 29), MASPCG_ERR_CAPACITY, "too many blocks");
  if (h->cfg.preconditioner == MASPCG_PRECOND_MAS32 || h->cfg.preconditioner == MASPCG_PRECOND_MAS16) {
    MREQ(h->has_graph, MASPCG_ERR_NOT_READY, "MAS needs set_graph before set_matrix_bcoo");
    MREQ(4LL * abd_body_count <= fem_offset_blocks, MASPCG_ERR_INVALID_ARGUMENT, "ABD rows overlap the FEM range");
    MREQ((long long)fem_offset_blocks + h->nv <= block_rows, MASPCG_ERR_INVALID_ARGUMENT,
         "FEM range exceeds block_rows");
  }
}

// The matrix build from device triplets (values may still be copying on the
// side stream: h->vals_pending).
void finish_set_matrix(maspcg_handle* h, const double* v, const int* r, const int* c, int n_blocks, int block_rows,
                       int fem_offset_blocks, int abd_body_count)
{
  h->nb = block_rows;
  h->fem_off = fem_offset_blocks;
  h->abd_bodies = abd_body_count;
  h->n_in = n_blocks;
  maspcg::build_internal_matrix(h, v, r, c, n_blocks);
  alloc_vectors(h);
  MCK(cudaStreamSynchronize(h->stream));
  h->has_matrix = true;
  h->has_precond = false;
  // no graph_dirty: the solve re-captures when the sizes or any buffer
  // changed (graph_signature)
}
}  // namespace

MASPCG_API maspcg_status maspcg_set_matrix_bcoo(maspcg_handle* h, const double* values9, const int* rows,
                                                const int* cols, int n_blocks, int block_rows, int fem_offset_blocks,
                                                int abd_body_count)
{
  return guard(h, [&] {
    check_matrix_args(h, n_blocks, block_rows, fem_offset_blocks, abd_body_count);
    const int* r = device_in(h, rows, (size_t)n_blocks, h->in_rows);
    const int* c = device_in(h, cols, (size_t)n_blocks, h->in_cols);
    // Host values (the bulk of the input) are copied on the side stream while
    // the structure is built from the indices; the value fill waits for them.
    const double* v = values9;
    h->vals_pending = false;
    MREQ(values9 != nullptr, MASPCG_ERR_INVALID_ARGUMENT, "null array argument");
    if (!is_device_ptr(values9)) {
      h->in_vals.resize((size_t)9 * n_blocks);
      MCK(cudaEventRecord(h->ev_fork, h->stream));  // earlier readers of in_vals are done
      MCK(cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0));
      MCK(cudaMemcpyAsync(h->in_vals.get(), values9, sizeof(double) * 9 * (size_t)n_blocks, cudaMemcpyHostToDevice,
                          h->side_stream));
      MCK(cudaEventRecord(h->ev_join, h->side_stream));
      h->vals_pending = true;
      v = h->in_vals.get();
    }
    finish_set_matrix(h, v, r, c, n_blocks, block_rows, fem_offset_blocks, abd_body_count);
  });
}

MASPCG_API maspcg_status maspcg_set_matrix_bcoo_indexed(maspcg_handle* h, const double* values9, const int* rows,
                                                        const int* cols, long long source_count,
                                                        const uint32_t* indices, int n_blocks, int offset,
                                                        int block_rows, int fem_offset_blocks, int abd_body_count)
{
  return guard(h, [&] {
    check_matrix_args(h, n_blocks, block_rows, fem_offset_blocks, abd_body_count);
    MREQ(source_count >= 1 && source_count <= (1LL << 31), MASPCG_ERR_INVALID_ARGUMENT, "bad source_count");
    MREQ(indices != nullptr || n_blocks <= source_count, MASPCG_ERR_INVALID_ARGUMENT,
         "without indices n_blocks must not exceed source_count");
    const double* sv = device_in(h, values9, 9 * (size_t)source_count, h->asm_vals);
    const int* sr = device_in(h, rows, (size_t)source_count, h->asm_rows);
    const int* sc = device_in(h, cols, (size_t)source_count, h->asm_cols);
    DBuf<unsigned> idx_stage{false};
    const unsigned* ix = indices ? device_in(h, (const unsigned*)indices, (size_t)n_blocks, idx_stage) : nullptr;
    h->in_vals.resize((size_t)9 * n_blocks);
    h->in_rows.resize((size_t)n_blocks);
    h->in_cols.resize((size_t)n_blocks);
    maspcg::gather_triplets(h, n_blocks, ix, sr, sc, sv, source_count, offset, h->in_rows.get(), h->in_cols.get(),
                            h->in_vals.get());
    h->vals_pending = false;
    finish_set_matrix(h, h->in_vals.get(), h->in_rows.get(), h->in_cols.get(), n_blocks, block_rows,
                      fem_offset_blocks, abd_body_count);
  });
}

MASPCG_API maspcg_status maspcg_build_preconditioner(maspcg_handle* h)
{
  return guard(h, [&] {
    MREQ(h->has_matrix, MASPCG_ERR_NOT_READY, "set_matrix_bcoo first");
    if (h->mas_layout) {
      maspcg::build_hierarchy(h);
      maspcg::build_mas_domains(h, nullptr);
    }
    maspcg::build_block_jacobi(h);
    MCK(cudaStreamSynchronize(h->stream));
    h->has_precond = true;
  });
}

MASPCG_API maspcg_status maspcg_refresh_matrix_values(maspcg_handle* h, const double* values9)
{
  return guard(h, [&] {
    MREQ(h->has_matrix && h->has_precond, MASPCG_ERR_NOT_READY, "set_matrix_bcoo and build_preconditioner first");
    MREQ(values9 != nullptr, MASPCG_ERR_INVALID_ARGUMENT, "null values");
    const double* v = device_in(h, values9, (size_t)9 * h->n_in, h->in_vals);
    maspcg::refresh_internal_values(h, v);
    if (h->mas_layout) maspcg::build_mas_domains(h, nullptr);
    maspcg::build_block_jacobi(h);
    MCK(cudaStreamSynchronize(h->stream));
  });
}

MASPCG_API maspcg_status maspcg_refresh_matrix_values_indexed(maspcg_handle* h, const double* values9,
                                                             long long source_count, const uint32_t* indices)
{
  return guard(h, [&] {
    MREQ(h->has_matrix && h->has_precond, MASPCG_ERR_NOT_READY, "set_matrix_bcoo and build_preconditioner first");
    MREQ(values9 != nullptr && indices != nullptr, MASPCG_ERR_INVALID_ARGUMENT, "null argument");
    MREQ(source_count >= 1 && source_count <= (1LL << 31), MASPCG_ERR_INVALID_ARGUMENT, "bad source_count");
    const std::vector<uint32_t> ix = host_copy(h, indices, (size_t)h->n_in);
    for (uint32_t t : ix) MREQ((long long)t < source_count, MASPCG_ERR_INVALID_ARGUMENT, "index past the source");
    const double* sv = device_in(h, values9, 9 * (size_t)source_count, h->asm_vals);
    DBuf<unsigned> idx_stage{false};
    const unsigned* id = device_in(h, (const unsigned*)indices, (size_t)h->n_in, idx_stage);
    h->in_vals.resize((size_t)9 * h->n_in);
    maspcg::gather_triplets(h, h->n_in, id, nullptr, nullptr, sv, source_count, 0, nullptr, nullptr,
                            h->in_vals.get());
    maspcg::refresh_internal_values(h, h->in_vals.get());
    if (h->mas_layout) maspcg::build_mas_domains(h, nullptr);
    maspcg::build_block_jacobi(h);
    MCK(cudaStreamSynchronize(h->stream));
  });
}

MASPCG_API maspcg_status maspcg_solve(maspcg_handle* h, const double* b, double* x, maspcg_result* out)
{
  return guard(h, [&] {
    MREQ(h->has_precond, MASPCG_ERR_NOT_READY, "build_preconditioner first");
    MREQ(b && x, MASPCG_ERR_INVALID_ARGUMENT, "null vector");
    const size_t n = 3 * (size_t)h->nb;
    const double* bd = device_in(h, b, n, h->io_a);
    maspcg::permute_in(h, bd, h->b64.get());
    maspcg::solve(h, h->b64.get(), h->io_b.get(), out);
    if (is_device_ptr(x)) {
      maspcg::permute_out(h, h->io_b.get(), x);
    } else {
      maspcg::permute_out(h, h->io_b.get(), h->io_a.get());
      MCK(cudaMemcpyAsync(x, h->io_a.get(), n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    }
    MCK(cudaStreamSynchronize(h->stream));
  });
}

MASPCG_API maspcg_status maspcg_apply_preconditioner(maspcg_handle* h, const double* r, double* z)
{
  return guard(h, [&] {
    MREQ(h->has_precond, MASPCG_ERR_NOT_READY, "build_preconditioner first");
    MREQ(r && z, MASPCG_ERR_INVALID_ARGUMENT, "null vector");
    const size_t n = 3 * (size_t)h->nb;
    const double* rd = device_in(h, r, n, h->io_a);
    maspcg::permute_in(h, rd, h->io_b.get());
    maspcg::apply_preconditioner64(h, h->io_b.get(), h->r64.get());
    if (is_device_ptr(z)) {
      maspcg::permute_out(h, h->r64.get(), z);
    } else {
      maspcg::permute_out(h, h->r64.get(), h->io_a.get());
      MCK(cudaMemcpyAsync(z, h->io_a.get(), n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    }
    MCK(cudaStreamSynchronize(h->stream));
  });
}

MASPCG_API maspcg_status maspcg_spmv(maspcg_handle* h, double a, const double* x, double b, double* y)
{
  return guard(h, [&] {
    MREQ(h->has_matrix, MASPCG_ERR_NOT_READY, "set_matrix_bcoo first");
    MREQ(x && y, MASPCG_ERR_INVALID_ARGUMENT, "null vector");
    const size_t n = 3 * (size_t)h->nb;
    const double* xd = device_in(h, x, n, h->io_a);
    maspcg::permute_in(h, xd, h->io_b.get());
    if (b != 0.0) {
      const double* yd = device_in(h, (const double*)y, n, h->io_a);
      maspcg::permute_in(h, yd, h->r64.get());
    }
    maspcg::launch_spmv64(h, h->io_b.get(), h->r64.get(), a, b);
    if (is_device_ptr(y)) {
      maspcg::permute_out(h, h->r64.get(), y);
    } else {
      maspcg::permute_out(h, h->r64.get(), h->io_a.get());
      MCK(cudaMemcpyAsync(y, h->io_a.get(), n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    }
    MCK(cudaStreamSynchronize(h->stream));
  });
}

MASPCG_API maspcg_status maspcg_spmv_working(maspcg_handle* h, const double* x, double* y)
{
  return guard(h, [&] {
    MREQ(h->has_matrix, MASPCG_ERR_NOT_READY, "set_matrix_bcoo first");
    MREQ(x && y, MASPCG_ERR_INVALID_ARGUMENT, "null vector");
    const size_t n = 3 * (size_t)h->nb;
    const double* xd = device_in(h, x, n, h->io_a);
    maspcg::permute_in(h, xd, h->io_b.get());
    maspcg::spmv_working(h, h->io_b.get(), h->r64.get());
    if (is_device_ptr(y)) {
      maspcg::permute_out(h, h->r64.get(), y);
    } else {
      maspcg::permute_out(h, h->r64.get(), h->io_a.get());
      MCK(cudaMemcpyAsync(y, h->io_a.get(), n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    }
    MCK(cudaStreamSynchronize(h->stream));
    h->graph_dirty = true;
  });
}

MASPCG_API maspcg_status maspcg_get_info(maspcg_handle* h, maspcg_info* info)
{
  return guard(h, [&] {
    MREQ(info, MASPCG_ERR_INVALID_ARGUMENT, "null info");
    maspcg_info i{};
    i.levelnum = h->levelnum;
    i.total_clusters = h->lv.total_clusters;
    i.domains = h->lv.domains;
    i.vert_num = h->nv;
    i.part_map_size = h->c0;
    i.going_next_capacity = h->gn_cap;
    i.internal_block_rows = h->nb_int;
    i.bcsr_blocks = h->nnzb;
    i.failed_domains = h->failed_domains;
    i.kernel_launches = h->kernel_launches;
    i.graph_captures = h->graph_captures;
    *info = i;
  });
}

MASPCG_API maspcg_status maspcg_get_hierarchy(maspcg_handle* h, uint32_t* fine_mask, int* cst, int* going_next,
                                              int* level_size, int* coarse_table, int* prefix_original)
{
  return guard(h, [&] {
    MREQ(h->has_precond && h->mas_layout, MASPCG_ERR_NOT_READY, "build a MAS preconditioner first");
    cudaStream_t s = h->stream;
    const size_t nv = h->nv;
    if (fine_mask) MCK(cudaMemcpyAsync(fine_mask, h->fine_mask.get(), nv * 4, cudaMemcpyDeviceToHost, s));
    if (cst) MCK(cudaMemcpyAsync(cst, h->cst.get(), nv * h->levelnum * 4, cudaMemcpyDeviceToHost, s));
    if (going_next)
      MCK(cudaMemcpyAsync(going_next, h->going_next.get(), (size_t)h->gn_cap * 4, cudaMemcpyDeviceToHost, s));
    if (level_size)
      MCK(cudaMemcpyAsync(level_size, h->level_size.get(), sizeof(int) * 2 * (h->levelnum + 1), cudaMemcpyDeviceToHost,
                          s));
    if (coarse_table) MCK(cudaMemcpyAsync(coarse_table, h->coarse_table.get(), nv * 6 * 4, cudaMemcpyDeviceToHost, s));
    if (prefix_original)
      MCK(cudaMemcpyAsync(prefix_original, h->prefix_orig.get(), (size_t)(h->c0 / h->bank) * 4, cudaMemcpyDeviceToHost,
                          s));
    MCK(cudaStreamSynchronize(s));
  });
}

MASPCG_API maspcg_status maspcg_get_bcsr(maspcg_handle* h, int* rowptr, int* colidx, double* values, int* internal_of_row)
{
  return guard(h, [&] {
    MREQ(h->has_matrix, MASPCG_ERR_NOT_READY, "set_matrix_bcoo first");
    cudaStream_t s = h->stream;
    if (rowptr) MCK(cudaMemcpyAsync(rowptr, h->rowptr.get(), sizeof(int) * (h->nb_int + 1), cudaMemcpyDeviceToHost, s));
    if (colidx) MCK(cudaMemcpyAsync(colidx, h->colidx.get(), sizeof(int) * h->nnzb, cudaMemcpyDeviceToHost, s));
    if (values)
      MCK(cudaMemcpyAsync(values, h->val64.get(), sizeof(double) * 9 * (size_t)h->nnzb, cudaMemcpyDeviceToHost, s));
    if (internal_of_row)
      MCK(cudaMemcpyAsync(internal_of_row, h->int_of_row.get(), sizeof(int) * h->nb, cudaMemcpyDeviceToHost, s));
    MCK(cudaStreamSynchronize(s));
  });
}

MASPCG_API maspcg_status maspcg_get_domain_inverses(maspcg_handle* h, float* out)
{
  return guard(h, [&] {
    MREQ(h->has_precond && h->mas_layout, MASPCG_ERR_NOT_READY, "build a MAS preconditioner first");
    MREQ(out, MASPCG_ERR_INVALID_ARGUMENT, "null output");
    maspcg::decode_inverses(h, out);
  });
}

MASPCG_API maspcg_status maspcg_get_domain_matrices(maspcg_handle* h, double* out)
{
  return guard(h, [&] {
    MREQ(h->has_precond && h->mas_layout, MASPCG_ERR_NOT_READY, "build a MAS preconditioner first");
    MREQ(out, MASPCG_ERR_INVALID_ARGUMENT, "null output");
    const size_t n = (size_t)h->lv.domains * (h->bank == 16 ? maspcg::kMas16Packed : maspcg::kPacked) * 9;
    DBuf<double> tmp{false};
    tmp.resize(n);
    MCK(cudaMemsetAsync(tmp.get(), 0, n * sizeof(double), h->stream));
    maspcg::gather_mas_domains(h, tmp.get());
    MCK(cudaMemcpyAsync(out, tmp.get(), n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    MCK(cudaStreamSynchronize(h->stream));
    h->graph_dirty = true;
  });
}

namespace {
// Runs the per-domain checks on device arrays and fills the caller's outputs.
void run_local_checks(maspcg_handle* h, int count, int bank, const double* p64, const float* i32,
                      maspcg_domain_check* per_domain, maspcg_diagnostics* summary)
{
  DBuf<double> res{false};
  res.resize(7 * (size_t)std::max(count, 1));
  maspcg::check_local_matrices(h, count, bank, p64, i32, res.get());
  std::vector<double> r(7 * (size_t)count);
  if (count) MCK(cudaMemcpyAsync(r.data(), res.get(), r.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  MCK(cudaStreamSynchronize(h->stream));
  maspcg_diagnostics d{};
  d.matrix_count = count;
  d.first_local_spd_failure = d.first_inverse_spd_failure = -1;
  d.minimum_local_diagonal = d.minimum_inverse_diagonal = std::numeric_limits<double>::infinity();
  for (int i = 0; i < count; ++i) {
    const double* o = &r[7 * (size_t)i];
    maspcg_domain_check c{};
    c.local_finite = o[0] != 0.0;
    c.inverse_finite = o[1] != 0.0;
    c.local_spd = o[2] != 0.0;
    c.inverse_spd = o[3] != 0.0;
    c.minimum_local_diagonal = o[4];
    c.minimum_inverse_diagonal = o[5];
    c.inverse_residual = o[6];
    if (per_domain) per_domain[i] = c;
    d.local_spd_count += c.local_spd;
    d.inverse_spd_count += c.inverse_spd;
    d.nonfinite_local_count += !c.local_finite;
    d.nonfinite_inverse_count += !c.inverse_finite;
    if (!c.local_spd && d.first_local_spd_failure < 0) d.first_local_spd_failure = i;
    if (!c.inverse_spd && d.first_inverse_spd_failure < 0) d.first_inverse_spd_failure = i;
    d.minimum_local_diagonal = std::min(d.minimum_local_diagonal, c.minimum_local_diagonal);
    d.minimum_inverse_diagonal = std::min(d.minimum_inverse_diagonal, c.minimum_inverse_diagonal);
    if (!std::isfinite(c.inverse_residual))
      d.maximum_inverse_residual = std::numeric_limits<double>::infinity();
    else
      d.maximum_inverse_residual = std::max(d.maximum_inverse_residual, c.inverse_residual);
  }
  d.passed = count > 0 && d.local_spd_count == count && d.inverse_spd_count == count && !d.nonfinite_local_count &&
             !d.nonfinite_inverse_count && d.maximum_inverse_residual <= 1e-3;
  if (summary) *summary = d;
}
}  // namespace

MASPCG_API maspcg_status maspcg_check_local_matrices(maspcg_handle* h, int count, int bank, const double* packed64,
                                                     const float* inverse32, maspcg_domain_check* per_domain,
                                                     maspcg_diagnostics* summary)
{
  return guard(h, [&] {
    MREQ(count >= 0, MASPCG_ERR_INVALID_ARGUMENT, "negative count");
    MREQ(bank == 32 || bank == 16, MASPCG_ERR_INVALID_ARGUMENT, "bank must be 32 or 16");
    const size_t per = (size_t)bank * (bank + 1) / 2 * 9;
    DBuf<double> a{false};
    DBuf<float> b{false};
    const double* pa = count ? device_in(h, packed64, per * count, a) : nullptr;
    const float* pb = count ? device_in(h, inverse32, per * count, b) : nullptr;
    run_local_checks(h, count, bank, pa, pb, per_domain, summary);
  });
}

MASPCG_API maspcg_status maspcg_local_diagnostics(maspcg_handle* h, maspcg_domain_check* per_domain,
                                                  maspcg_diagnostics* summary)
{
  return guard(h, [&] {
    MREQ(h->has_precond && h->mas_layout, MASPCG_ERR_NOT_READY, "build a MAS preconditioner first");
    const int D = h->lv.domains;
    const size_t per = (size_t)(h->bank == 16 ? maspcg::kMas16Packed : maspcg::kPacked) * 9;
    DBuf<double> a{false};
    a.resize(per * std::max(D, 1));
    MCK(cudaMemsetAsync(a.get(), 0, per * D * sizeof(double), h->stream));
    maspcg::gather_mas_domains(h, a.get());
    std::vector<float> inv(per * D);
    maspcg::decode_inverses(h, inv.data());
    DBuf<float> b{false};
    b.resize(per * std::max(D, 1));
    MCK(cudaMemcpyAsync(b.get(), inv.data(), inv.size() * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    run_local_checks(h, D, h->bank, a.get(), b.get(), per_domain, summary);
    h->graph_dirty = true;
  });
}

MASPCG_API maspcg_status maspcg_time_stage(maspcg_handle* h, int stage, int repeats, double* mean_ms)
{
  return guard(h, [&] {
    MREQ(h->has_precond, MASPCG_ERR_NOT_READY, "build_preconditioner first");
    MREQ(mean_ms && repeats >= 1, MASPCG_ERR_INVALID_ARGUMENT, "bad arguments");
    *mean_ms = maspcg::time_stage(h, stage, repeats);
    h->graph_dirty = true;
  });
}

MASPCG_API maspcg_status maspcg_set_wait_test_hooks(maspcg_handle* h, long long barrier_limit, int barrier_extra)
{
  return guard(h, [&] {
    MREQ(barrier_limit >= 1 && barrier_extra >= 0 && barrier_extra <= 1024, MASPCG_ERR_INVALID_ARGUMENT,
         "barrier_limit >= 1, 0 <= barrier_extra <= 1024");
    h->barrier_limit = barrier_limit;
    h->barrier_extra = barrier_extra;
  });
}

MASPCG_API maspcg_status maspcg_bcoo_gradient(maspcg_handle* h, const int* rows, const int* cols, int n_blocks,
                                              const double* lam, const double* x, double* grad9)
{
  return guard(h, [&] {
    MREQ(h->has_matrix, MASPCG_ERR_NOT_READY, "set_matrix_bcoo first");
    MREQ(n_blocks >= 0, MASPCG_ERR_INVALID_ARGUMENT, "negative block count");
    if (n_blocks == 0) return;
    MREQ(rows && cols && lam && x && grad9, MASPCG_ERR_INVALID_ARGUMENT, "null argument");
    const size_t n = 3 * (size_t)h->nb;
    const int* r = device_in(h, rows, (size_t)n_blocks, h->adj_rows);
    const int* c = device_in(h, cols, (size_t)n_blocks, h->adj_cols);
    // block indices must address the system (checked on the host copy)
    {
      const std::vector<int> hr = host_copy(h, rows, (size_t)n_blocks), hc = host_copy(h, cols, (size_t)n_blocks);
      for (int t = 0; t < n_blocks; ++t)
        MREQ(hr[t] >= 0 && hr[t] < h->nb && hc[t] >= 0 && hc[t] < h->nb, MASPCG_ERR_INVALID_ARGUMENT,
             "block index outside the system");
    }
    const double* l = device_in(h, lam, n, h->adj_lam);
    const double* xv = device_in(h, x, n, h->adj_x);
    if (is_device_ptr(grad9)) {
      maspcg::bcoo_gradient(h, r, c, n_blocks, l, xv, grad9);
    } else {
      h->adj_grad.resize((size_t)9 * n_blocks);
      maspcg::bcoo_gradient(h, r, c, n_blocks, l, xv, h->adj_grad.get());
      MCK(cudaMemcpyAsync(grad9, h->adj_grad.get(), sizeof(double) * 9 * (size_t)n_blocks, cudaMemcpyDeviceToHost,
                          h->stream));
    }
    MCK(cudaStreamSynchronize(h->stream));
  });
}

MASPCG_API maspcg_status maspcg_element_modulus_gradient(maspcg_handle* h, int n_tets, int blocks_per_tet,
                                                         const int* rows, const int* cols, const double* values9,
                                                         const double* lam, const double* x, const double* youngs,
                                                         double* grad_youngs)
{
  return guard(h, [&] {
    MREQ(h->has_matrix, MASPCG_ERR_NOT_READY, "set_matrix_bcoo first");
    MREQ(n_tets >= 0 && blocks_per_tet >= 1 && blocks_per_tet <= 64, MASPCG_ERR_INVALID_ARGUMENT,
         "n_tets >= 0, 1 <= blocks_per_tet <= 64");
    if (n_tets == 0) return;
    MREQ(rows && cols && values9 && lam && x && youngs && grad_youngs, MASPCG_ERR_INVALID_ARGUMENT, "null argument");
    const size_t nblk = (size_t)n_tets * blocks_per_tet;
    MREQ(nblk <= (size_t)0x7fffffff, MASPCG_ERR_CAPACITY, "too many blocks");
    {
      const std::vector<int> hr = host_copy(h, rows, nblk), hc = host_copy(h, cols, nblk);
      for (size_t t = 0; t < nblk; ++t)
        MREQ(hr[t] >= 0 && hr[t] < h->nb && hc[t] >= 0 && hc[t] < h->nb, MASPCG_ERR_INVALID_ARGUMENT,
             "block index outside the system");
    }
    const size_t n = 3 * (size_t)h->nb;
    const int* r = device_in(h, rows, nblk, h->adj_rows);
    const int* c = device_in(h, cols, nblk, h->adj_cols);
    DBuf<double> vstage{false}, estage{false};
    const double* v = device_in(h, values9, 9 * nblk, vstage);
    const double* l = device_in(h, lam, n, h->adj_lam);
    const double* xv = device_in(h, x, n, h->adj_x);
    const double* e = device_in(h, youngs, (size_t)n_tets, estage);
    DBuf<double> gstage{false};
    double* g = device_out(grad_youngs, (size_t)n_tets, gstage);
    maspcg::modulus_gradient(h, r, c, v, n_tets, blocks_per_tet, l, xv, e, g);
    copy_back(h, grad_youngs, (const double*)g, (size_t)n_tets);
    MCK(cudaStreamSynchronize(h->stream));
  });
}

MASPCG_API maspcg_status maspcg_convert_bcoo(maspcg_handle* h, const double* values9, const int* rows,
                                             const int* cols, int n, double* values9_out, int* rows_out,
                                             int* cols_out, int* n_out)
{
  return guard(h, [&] {
    MREQ(n >= 0, MASPCG_ERR_INVALID_ARGUMENT, "negative triplet count");
    MREQ(n_out != nullptr, MASPCG_ERR_INVALID_ARGUMENT, "null n_out");
    *n_out = 0;
    if (n == 0) return;
    MREQ(values9_out && rows_out && cols_out, MASPCG_ERR_INVALID_ARGUMENT, "null output array");
    const double* v = device_in(h, values9, (size_t)9 * n, h->asm_vals);
    const int* r = device_in(h, rows, (size_t)n, h->asm_rows);
    const int* c = device_in(h, cols, (size_t)n, h->asm_cols);
    double* vo = device_out(values9_out, (size_t)9 * n, h->asm_vals_out);
    int* ro = device_out(rows_out, (size_t)n, h->asm_rows_out);
    int* co = device_out(cols_out, (size_t)n, h->asm_cols_out);
    const int count = maspcg::convert_bcoo(h, r, c, v, n, ro, co, vo);
    copy_back(h, values9_out, vo, (size_t)9 * count);
    copy_back(h, rows_out, ro, (size_t)count);
    copy_back(h, cols_out, co, (size_t)count);
    MCK(cudaStreamSynchronize(h->stream));
    *n_out = count;
  });
}

MASPCG_API maspcg_status maspcg_partition_contact_triplets(maspcg_handle* h, const double* values9, const int* rows,
                                                           const int* cols, const unsigned long long* type_hash,
                                                           int n, double* values9_out, int* rows_out,
                                                           int* cols_out, int counts[4])
{
  return guard(h, [&] {
    MREQ(n >= 0, MASPCG_ERR_INVALID_ARGUMENT, "negative triplet count");
    MREQ(counts != nullptr, MASPCG_ERR_INVALID_ARGUMENT, "null counts");
    counts[0] = counts[1] = counts[2] = counts[3] = 0;
    if (n == 0) return;
    MREQ(values9_out && rows_out && cols_out, MASPCG_ERR_INVALID_ARGUMENT, "null output array");
    const double* v = device_in(h, values9, (size_t)9 * n, h->asm_vals);
    const int* r = device_in(h, rows, (size_t)n, h->asm_rows);
    const int* c = device_in(h, cols, (size_t)n, h->asm_cols);
    const unsigned long long* t = device_in(h, type_hash, (size_t)n, h->asm_types);
    double* vo = device_out(values9_out, (size_t)9 * n, h->asm_vals_out);
    int* ro = device_out(rows_out, (size_t)n, h->asm_rows_out);
    int* co = device_out(cols_out, (size_t)n, h->asm_cols_out);
    int k[4];
    maspcg::partition_contacts(h, r, c, v, t, n, ro, co, vo, k);
    copy_back(h, values9_out, vo, (size_t)9 * n);
    copy_back(h, rows_out, ro, (size_t)n);
    copy_back(h, cols_out, co, (size_t)n);
    MCK(cudaStreamSynchronize(h->stream));
    for (int q = 0; q < 4; ++q) counts[q] = k[q];
  });
}


MASPCG_API maspcg_status maspcg_adjust_contact_triplets(maspcg_handle* h, int n, int* rows, int* cols,
                                                        double* values9_colmajor, const int* bd_type, int n_vertices,
                                                        int fem_offset)
{
  return triplet_fixup(h, n, rows, cols, values9_colmajor, bd_type, n_vertices, fem_offset, false);
}

MASPCG_API maspcg_status maspcg_zero_boundary_triplets(maspcg_handle* h, int n, const int* rows, const int* cols,
                                                       double* values9_colmajor, const int* bd_type, int n_vertices,
                                                       int index_offset)
{
  return triplet_fixup(h, n, const_cast<int*>(rows), const_cast<int*>(cols), values9_colmajor, bd_type, n_vertices,
                       index_offset, true);
}

MASPCG_API maspcg_status maspcg_fem_snk1_gradient_hessian(maspcg_handle* h, int n_tets, const unsigned* tets,
                                                          int n_vertices, const double* x, const double* dm_inverse,
                                                          const double* volume, const double* len_rate,
                                                          const double* vol_rate, double dt, int hessian_offset,
                                                          double* gradient, int* rows, int* cols,
                                                          double* values9_colmajor)
{
  return guard(h, [&] {
    MREQ(n_tets >= 0 && n_vertices >= 0, MASPCG_ERR_INVALID_ARGUMENT, "negative count");
    MREQ(std::isfinite(dt), MASPCG_ERR_INVALID_ARGUMENT, "non-finite dt");
    if (n_tets == 0) return;
    MREQ(gradient && rows && cols && values9_colmajor, MASPCG_ERR_INVALID_ARGUMENT, "null output array");
    MREQ((long long)hessian_offset + n_vertices <= 0x7fffffffLL && hessian_offset >= 0, MASPCG_ERR_CAPACITY,
         "block index overflow");
    MREQ(10LL * n_tets <= 0x7fffffffLL, MASPCG_ERR_CAPACITY, "too many tets");
    const unsigned* td = device_in(h, tets, 4 * (size_t)n_tets, h->fem_tets);
    const double* xd = device_in(h, x, 3 * (size_t)n_vertices, h->fem_x);
    const double* di = device_in(h, dm_inverse, 9 * (size_t)n_tets, h->fem_dminv);
    const double* vo = device_in(h, volume, (size_t)n_tets, h->fem_vol);
    const double* lr = device_in(h, len_rate, (size_t)n_tets, h->fem_len);
    const double* vr = device_in(h, vol_rate, (size_t)n_tets, h->fem_volr);
    const bool dev = is_device_ptr(gradient);
    double* gd = gradient;
    if (!dev) {
      h->fem_grad.resize(3 * (size_t)n_vertices);
      gd = h->fem_grad.get();
      MCK(cudaMemcpyAsync(gd, gradient, sizeof(double) * 3 * (size_t)n_vertices, cudaMemcpyHostToDevice, h->stream));
    }
    int* ro = device_out(rows, 10 * (size_t)n_tets, h->asm_rows_out);
    int* co = device_out(cols, 10 * (size_t)n_tets, h->asm_cols_out);
    double* va = device_out(values9_colmajor, 90 * (size_t)n_tets, h->asm_vals_out);
    maspcg::fem_snk1(h, n_tets, n_vertices, td, xd, di, vo, lr, vr, dt, hessian_offset, gd, ro, co, va);
    if (!dev) copy_back(h, gradient, gd, 3 * (size_t)n_vertices);
    copy_back(h, rows, ro, 10 * (size_t)n_tets);
    copy_back(h, cols, co, 10 * (size_t)n_tets);
    copy_back(h, values9_colmajor, va, 90 * (size_t)n_tets);
    MCK(cudaStreamSynchronize(h->stream));
  });
}

MASPCG_API maspcg_status maspcg_galerkin_coarse_matrix(maspcg_handle* h, const maspcg_galerkin_map* map,
                                                       const double* values9, const int* rows, const int* cols,
                                                       int n, double* coarse_values9, int* coarse_rows,
                                                       int* coarse_cols, int capacity, int* n_coarse)
{
  return guard(h, [&] {
    MREQ(n >= 0 && capacity >= 0, MASPCG_ERR_INVALID_ARGUMENT, "negative count");
    MREQ(n_coarse != nullptr, MASPCG_ERR_INVALID_ARGUMENT, "null n_coarse");
    *n_coarse = 0;
    const maspcg::GalerkinMap m = galerkin_map(h, map);
    if (n == 0) return;
    const double* v = device_in(h, values9, (size_t)9 * n, h->gal_in_vals);
    const int* r = device_in(h, rows, (size_t)n, h->gal_in_rows);
    const int* c = device_in(h, cols, (size_t)n, h->gal_in_cols);
    const double* ev;
    const int *er, *ec;
    const int expanded = maspcg::galerkin_expand(h, m, v, r, c, n, &ev, &er, &ec);
    h->gal_out_vals.resize(9 * (size_t)std::max(expanded, 1));
    h->gal_out_rows.resize((size_t)std::max(expanded, 1));
    h->gal_out_cols.resize((size_t)std::max(expanded, 1));
    const int count = maspcg::convert_bcoo(h, er, ec, ev, expanded, h->gal_out_rows.get(), h->gal_out_cols.get(),
                                           h->gal_out_vals.get());
    *n_coarse = count;
    MREQ(count <= capacity, MASPCG_ERR_CAPACITY,
         "coarse output holds " + std::to_string(capacity) + " blocks, " + std::to_string(count) + " needed");
    MREQ(count == 0 || (coarse_values9 && coarse_rows && coarse_cols), MASPCG_ERR_INVALID_ARGUMENT,
         "null output array");
    const cudaMemcpyKind kind = cudaMemcpyDefault;
    MCK(cudaMemcpyAsync(coarse_values9, h->gal_out_vals.get(), sizeof(double) * 9 * (size_t)count, kind, h->stream));
    MCK(cudaMemcpyAsync(coarse_rows, h->gal_out_rows.get(), sizeof(int) * (size_t)count, kind, h->stream));
    MCK(cudaMemcpyAsync(coarse_cols, h->gal_out_cols.get(), sizeof(int) * (size_t)count, kind, h->stream));
    MCK(cudaStreamSynchronize(h->stream));
  });
}

MASPCG_API maspcg_status maspcg_galerkin_restrict(maspcg_handle* h, const maspcg_galerkin_map* map,
                                                  const double* fine_rhs, double* coarse_rhs)
{
  return guard(h, [&] {
    const maspcg::GalerkinMap m = galerkin_map(h, map);
    const int cb = map->prefix_blocks + map->coarse_block_nodes;
    if (cb == 0) return;
    MREQ(coarse_rhs != nullptr, MASPCG_ERR_INVALID_ARGUMENT, "null output array");
    const double* f = m.fine_blocks ? device_in(h, fine_rhs, 3 * (size_t)m.fine_blocks, h->gal_vec_in) : nullptr;
    double* o = device_out(coarse_rhs, 3 * (size_t)cb, h->gal_vec_out);
    maspcg::galerkin_restrict(h, m, f, o, cb);
    copy_back(h, coarse_rhs, o, 3 * (size_t)cb);
    MCK(cudaStreamSynchronize(h->stream));
  });
}

MASPCG_API maspcg_status maspcg_galerkin_prolong(maspcg_handle* h, const maspcg_galerkin_map* map,
                                                 const double* coarse_x, double* fine_x)
{
  return guard(h, [&] {
    const maspcg::GalerkinMap m = galerkin_map(h, map);
    if (m.fine_blocks == 0) return;
    MREQ(fine_x != nullptr, MASPCG_ERR_INVALID_ARGUMENT, "null output array");
    const int cb = map->prefix_blocks + map->coarse_block_nodes;
    const double* cx = device_in(h, coarse_x, 3 * (size_t)cb, h->gal_vec_in);
    double* o = device_out(fine_x, 3 * (size_t)m.fine_blocks, h->gal_vec_out);
    maspcg::galerkin_prolong(h, m, cx, o);
    copy_back(h, fine_x, o, 3 * (size_t)m.fine_blocks);
    MCK(cudaStreamSynchronize(h->stream));
  });
}

MASPCG_API maspcg_status maspcg_residual_norms_noalloc(maspcg_handle* h, int count, const double* x, const double* b,
                                                       double* residual_norms, double* rhs_norms)
{
  return guard(h, [&] {
    MREQ(h->has_matrix, MASPCG_ERR_NOT_READY, "set_matrix_bcoo first");
    MREQ(count >= 1 && count <= MASPCG_RESIDUAL_MAX_VECTORS, MASPCG_ERR_CAPACITY,
         "count must be 1.." + std::to_string(MASPCG_RESIDUAL_MAX_VECTORS) +
             ": the fixed scratch holds partial sums for that many vectors");
    MREQ(x && b && residual_norms, MASPCG_ERR_INVALID_ARGUMENT, "null argument");
    MREQ(is_device_ptr(x) && is_device_ptr(b), MASPCG_ERR_INVALID_ARGUMENT,
         "x and b must be device pointers: this entry point stages nothing");
    maspcg::residual_norms_noalloc(h, count, x, b, residual_norms, rhs_norms);
  });
}

}  // extern "C"
