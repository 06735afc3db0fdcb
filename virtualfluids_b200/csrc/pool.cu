// Domain pools (include/vfb.h, section 2c): many independent boxes in one device arena, advanced
// together by one persistent launch per step over a work list of node blocks.
//
// Host side only: the arena allocator, the domain table and work list, CUDA-graph replay of the
// step loop and the launch-shape autotuner. The kernel is k17_pool_kernel (kernels.cuh); domain
// initialisation and field output reuse the structured-box kernels on the domain's slice of the
// arena, so a domain computes exactly what a vfb_box of the same description computes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "guards.h"
#include "launch.h"
#include "pool_tables.h"
#include "vfb.h"

namespace {

int pool_fail(int status, const char *msg)
{
    vfb::set_last_error(msg);
    return status;
}

int pool_cuda(cudaError_t e, const char *what)
{
    if (e == cudaSuccess)
        return VFB_OK;
    const std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    vfb::set_last_error(m.c_str());
    return e == cudaErrorMemoryAllocation ? VFB_ERR_OUT_OF_MEMORY : VFB_ERR_CUDA;
}

size_t storage_size(int s) { return s == VFB_STORAGE_F64 ? 8 : s == VFB_STORAGE_F32 ? 4 : 2; }
size_t real_size(int s) { return s == VFB_STORAGE_F64 ? 8 : 4; }
constexpr uint64_t kAlign = 256;
uint64_t align_up(uint64_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// the launchers of one (storage, arithmetic) variant
struct PoolOps {
    cudaError_t (*collide)(void *, const void *, const uint2 *, const uint32_t *, int, bool, unsigned, unsigned,
                           cudaStream_t);
    const void *(*kernel)(bool);
    size_t (*domain_bytes)();
    void (*domain)(void *, const vfb::PoolDomainSpec &);
    cudaError_t (*bcs)(void *, const void *, const uint2 *, const uint32_t *, const uint2 *, const uint32_t *,
                       const uint2 *, const uint32_t *, bool, unsigned, cudaStream_t);
    cudaError_t (*mass)(void *, const void *, const uint2 *, uint32_t, int, int, bool, double *, cudaStream_t);
    cudaError_t (*init)(const vfb::BoxState &, bool, const void *, const void *, const void *, const void *,
                        cudaStream_t);
    cudaError_t (*macros)(const vfb::BoxState &, bool, void *, void *, void *, void *, cudaStream_t);
};

template <class LA>
PoolOps ops_of()
{
    return PoolOps{ LA::pool_collide, LA::pool_kernel, LA::pool_domain_bytes, LA::pool_domain, LA::pool_bcs,
                    LA::pool_mass, LA::box_init, LA::box_macros };
}

bool select_ops(int storage, int arith, PoolOps &out)
{
    if (arith == VFB_ARITH_EXACT) {
        if (storage == VFB_STORAGE_F64) { out = ops_of<vfb::exact::Launchers<double>>(); return true; }
        if (storage == VFB_STORAGE_F32) { out = ops_of<vfb::exact::Launchers<float>>(); return true; }
        return false;
    }
    switch (storage) {
    case VFB_STORAGE_F64: out = ops_of<vfb::fast::Launchers<double>>(); return true;
    case VFB_STORAGE_F32: out = ops_of<vfb::fast::Launchers<float>>(); return true;
    case VFB_STORAGE_F16: out = ops_of<vfb::fast::Launchers<__half>>(); return true;
    case VFB_STORAGE_BF16: out = ops_of<vfb::fast::Launchers<__nv_bfloat16>>(); return true;
    case VFB_STORAGE_E3M12: out = ops_of<vfb::fast::Launchers<vfb::e3m12_t>>(); return true;
    default: return false;
    }
}

// first-fit allocator over [0, size) in kAlign units, coalescing on release
class ArenaAllocator {
public:
    explicit ArenaAllocator(uint64_t size = 0) { if (size) free_[0] = size; }
    bool take(uint64_t bytes, uint64_t &offset)
    {
        bytes = align_up(bytes);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes)
                continue;
            offset = it->first;
            const uint64_t rest = it->second - bytes;
            free_.erase(it);
            if (rest)
                free_[offset + bytes] = rest;
            used_ += bytes;
            return true;
        }
        return false;
    }
    void give(uint64_t offset, uint64_t bytes)
    {
        bytes = align_up(bytes);
        used_ -= bytes;
        auto it = free_.emplace(offset, bytes).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }
    uint64_t used() const { return used_; }

private:
    std::map<uint64_t, uint64_t> free_;
    uint64_t used_ = 0;
};

struct DomainSlot {
    bool live = false, active = false;
    bool retired = false;          // removed, arena range not yet reusable (kernels may be in flight)
    vfb_domain_desc desc{};
    uint64_t nodes = 0, pitch = 0;
    uint64_t dist_offset = 0;      // bytes
    uint64_t mask_offset = 0;      // bytes
    uint64_t bytes = 0;            // bytes taken (populations, mask, boundary conditions)
    bool has_mask = false;
    uint32_t n_noslip = 0, n_pressure = 0;
    uint32_t n_guarded = 0;        // no-slip nodes with guarded directions
    double ref_mass = 0.0;         // watchdog: the mass at the first check after the initialisation
    bool has_ref = false;
};

// a work list on the device: {domain, first node} items and their count (a device word, so that a
// captured step keeps working after the list changes)
struct DeviceList {
    uint2 *items = nullptr;
    uint32_t *count = nullptr;
    size_t capacity = 0;
};

constexpr uint32_t kBCSpan = 128;   // BC nodes per item (one thread each)

constexpr uint32_t kGraphSteps = 16;

} // namespace

struct vfb_pool {
    vfb_pool_desc desc{};
    PoolOps ops{};
    void *arena = nullptr;
    ArenaAllocator alloc;
    std::vector<DomainSlot> slots;
    void *domain_table = nullptr;      // max_domains records in the compute type
    size_t record_bytes = 0;
    uint2 *items = nullptr;
    uint32_t *n_items = nullptr;
    size_t items_capacity = 0;
    bool list_dirty = true;
    uint64_t active_nodes = 0;
    bool even = true;
    int threads = 128, nodes_per_thread = 8, blocks_per_sm = -1, use_graph = 1;  // the default launch shape
    unsigned grid = 0;
    cudaGraphExec_t graph = nullptr;
    cudaStream_t graph_stream = nullptr;
    uint64_t launches = 0;
    void *staging = nullptr;           // host<->device field staging, outside the arena
    uint64_t staging_bytes = 0;
    DeviceList noslip_list, pressure_list;   // BC work lists of the active domains
    DeviceList guard_list;                   // the guarded no-slip nodes of the active domains
    bool has_noslip = false, has_pressure = false, has_guard = false;
    unsigned bc_grid = 0;
    std::vector<uint2> host_items;     // the collision work list as uploaded (watchdog sums)
    double *mass_partials = nullptr;   // one FP64 partial per work item
    size_t mass_capacity = 0;
};

namespace {

void drop_graph(vfb_pool *p)
{
    if (p->graph)
        cudaGraphExecDestroy(p->graph);
    p->graph = nullptr;
    p->graph_stream = nullptr;
}

int sm_count_here()
{
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 1;
}

cudaError_t update_grid(vfb_pool *p)
{
    if (p->blocks_per_sm < 0) {
        // one block per work item, no persistent loop: the grid follows the list's item count
        const unsigned g = (unsigned)std::max<size_t>(p->host_items.size(), 1);
        if (g != p->grid)
            drop_graph(p);
        p->grid = g;
        p->bc_grid = (unsigned)(4 * sm_count_here());
        return cudaSuccess;
    }
    int bps = p->blocks_per_sm;
    int occ = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, p->ops.kernel(true), p->threads, 0);
    if (e != cudaSuccess)
        return e;
    if (bps <= 0 || bps > occ)
        bps = std::max(1, occ);
    const unsigned g = (unsigned)(bps * sm_count_here());
    if (g != p->grid)
        drop_graph(p);
    p->grid = g;
    p->bc_grid = (unsigned)(4 * sm_count_here());
    return cudaSuccess;
}

// after the pool's stream has drained: the ranges and slots of removed domains become reusable
void reclaim(vfb_pool *p)
{
    for (DomainSlot &d : p->slots)
        if (d.retired) {
            p->alloc.give(d.dist_offset, d.bytes);
            d = DomainSlot();
        }
}

// copies `items` into a device list, growing it (and dropping the captured steps that refer to the
// old buffer) when needed; synchronous with respect to the host
cudaError_t upload_list(vfb_pool *p, DeviceList &L, const std::vector<uint2> &items, cudaStream_t s)
{
    cudaError_t e = cudaSuccess;
    if (!L.count) {
        e = cudaMalloc((void **)&L.count, sizeof(uint32_t));
        if (e != cudaSuccess)
            return e;
    }
    if (items.size() > L.capacity) {
        drop_graph(p);
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess)
            return e;
        cudaFree(L.items);
        L.items = nullptr;
        const size_t cap = std::max<size_t>(items.size() + items.size() / 2, 1024);
        e = cudaMalloc((void **)&L.items, cap * sizeof(uint2));
        L.capacity = e == cudaSuccess ? cap : 0;
        if (e != cudaSuccess)
            return e;
    }
    if (!items.empty())
        e = cudaMemcpyAsync(L.items, items.data(), items.size() * sizeof(uint2), cudaMemcpyHostToDevice, s);
    const uint32_t n = (uint32_t)items.size();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(L.count, &n, sizeof(uint32_t), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    return e;
}

// the boundary-condition work lists: per active domain with BC nodes one item per kBCSpan nodes
cudaError_t rebuild_bc_lists(vfb_pool *p, cudaStream_t s)
{
    std::vector<uint2> ns, pr, gd;
    for (uint32_t id = 0; id < p->slots.size(); ++id) {
        const DomainSlot &d = p->slots[id];
        if (!d.live || !d.active)
            continue;
        for (uint32_t i = 0; i < d.n_noslip; i += kBCSpan)
            ns.push_back(make_uint2(id, i));
        for (uint32_t i = 0; i < d.n_guarded; i += kBCSpan)
            gd.push_back(make_uint2(id, i));
        for (uint32_t i = 0; i < d.n_pressure; i += kBCSpan)
            pr.push_back(make_uint2(id, i));
    }
    const bool has_ns = !ns.empty(), has_pr = !pr.empty(), has_gd = !gd.empty();
    if (has_ns != p->has_noslip || has_pr != p->has_pressure || has_gd != p->has_guard)
        drop_graph(p);              // the launches of a step change
    p->has_noslip = has_ns;
    p->has_pressure = has_pr;
    p->has_guard = has_gd;
    cudaError_t e = cudaSuccess;
    if (has_ns || p->noslip_list.count)
        e = upload_list(p, p->noslip_list, ns, s);
    if (e == cudaSuccess && (has_gd || p->guard_list.count))
        e = upload_list(p, p->guard_list, gd, s);
    if (e == cudaSuccess && (has_pr || p->pressure_list.count))
        e = upload_list(p, p->pressure_list, pr, s);
    return e;
}

// the work list: per active domain (in id order) one item per `threads * nodes_per_thread` nodes
cudaError_t rebuild_list(vfb_pool *p, cudaStream_t s)
{
    const uint64_t span = (uint64_t)p->threads * (uint64_t)p->nodes_per_thread;
    std::vector<uint2> items;
    uint64_t nodes = 0;
    for (uint32_t id = 0; id < p->slots.size(); ++id) {
        const DomainSlot &d = p->slots[id];
        if (!d.live || !d.active)
            continue;
        nodes += d.nodes;
        for (uint64_t l0 = 0; l0 < d.nodes; l0 += span)
            items.push_back(make_uint2(id, (unsigned)l0));
    }
    cudaError_t e = cudaSuccess;
    if (items.size() > p->items_capacity) {
        // a new buffer: a captured step refers to the old one
        drop_graph(p);
        e = cudaStreamSynchronize(s);
        if (e == cudaSuccess) {
            cudaFree(p->items);
            p->items = nullptr;
            const size_t cap = std::max<size_t>(items.size() + items.size() / 2, 1024);
            e = cudaMalloc((void **)&p->items, cap * sizeof(uint2));
            p->items_capacity = e == cudaSuccess ? cap : 0;
        }
    }
    // the host vectors die with this call: copy synchronously with respect to the host
    if (e == cudaSuccess && !items.empty())
        e = cudaMemcpyAsync(p->items, items.data(), items.size() * sizeof(uint2), cudaMemcpyHostToDevice, s);
    const uint32_t n = (uint32_t)items.size();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p->n_items, &n, sizeof(uint32_t), cudaMemcpyHostToDevice, s);
    p->host_items = items;
    if (e == cudaSuccess && p->blocks_per_sm < 0)
        e = update_grid(p);        // a captured step's grid is the old item count
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e == cudaSuccess)
        e = rebuild_bc_lists(p, s);
    if (e == cudaSuccess)
        reclaim(p);
    p->active_nodes = nodes;
    p->list_dirty = false;
    return e;
}

// one step: the collision, then the no-slip BCs at its parity and the pressure BCs after the swap
cudaError_t launch_step(vfb_pool *p, bool even, cudaStream_t s)
{
    ++p->launches;
    cudaError_t e = p->ops.collide(p->arena, p->domain_table, p->items, p->n_items, p->nodes_per_thread, even, p->grid,
                                   (unsigned)p->threads, s);
    if (e == cudaSuccess && (p->has_noslip || p->has_pressure)) {
        p->launches += (p->has_noslip ? 1 : 0) + (p->has_guard ? 1 : 0) + (p->has_pressure ? 1 : 0);
        e = p->ops.bcs(p->arena, p->domain_table, p->has_noslip ? p->noslip_list.items : nullptr,
                       p->noslip_list.count, p->has_guard ? p->guard_list.items : nullptr, p->guard_list.count,
                       p->has_pressure ? p->pressure_list.items : nullptr, p->pressure_list.count, even, p->bc_grid,
                       s);
    }
    return e;
}

uint32_t launches_per_step(const vfb_pool *p)
{
    return 1u + (p->has_noslip ? 1u : 0u) + (p->has_guard ? 1u : 0u) + (p->has_pressure ? 1u : 0u);
}

// kGraphSteps steps starting at the even parity, captured once and replayed
cudaError_t ensure_graph(vfb_pool *p, cudaStream_t s)
{
    if (p->graph && p->graph_stream == s)
        return cudaSuccess;
    drop_graph(p);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess)
        return e;
    const uint64_t launches = p->launches;
    for (uint32_t i = 0; i < kGraphSteps; ++i)
        launch_step(p, (i & 1u) == 0, s);
    p->launches = launches;       // counted when the graph runs
    e = cudaStreamEndCapture(s, &g);
    if (e != cudaSuccess)
        return e;
    e = cudaGraphInstantiate(&p->graph, g, 0);
    cudaGraphDestroy(g);
    if (e == cudaSuccess)
        p->graph_stream = s;
    else
        p->graph = nullptr;
    return e;
}

// a staging buffer of at least `bytes` (grown only when a larger domain than any before is staged)
cudaError_t ensure_staging(vfb_pool *p, uint64_t bytes, cudaStream_t s)
{
    if (bytes <= p->staging_bytes)
        return cudaSuccess;
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return e;
    cudaFree(p->staging);
    p->staging = nullptr;
    p->staging_bytes = 0;
    const uint64_t want = bytes + bytes / 4;
    e = cudaMalloc(&p->staging, want);
    if (e == cudaSuccess)
        p->staging_bytes = want;
    return e;
}

vfb::BoxState domain_box(const vfb_pool *p, const DomainSlot &d)
{
    vfb::BoxState b{};
    b.dist = static_cast<char *>(p->arena) + d.dist_offset;
    b.pitch = d.pitch;
    b.nx = d.desc.nx;
    b.ny = d.desc.ny;
    b.nz = d.desc.nz;
    b.periodic_x = d.desc.periodic_x;
    b.periodic_y = d.desc.periodic_y;
    b.periodic_z = d.desc.periodic_z;
    b.mask = d.has_mask ? static_cast<const uint8_t *>(p->arena) + d.mask_offset : nullptr;
    b.omega = d.desc.omega;
    b.fx = d.desc.forces[0] * 0.5;
    b.fy = d.desc.forces[1] * 0.5;
    b.fz = d.desc.forces[2] * 0.5;
    for (int i = 0; i < 3; ++i)
        b.lim[i] = d.desc.quadric_limiters[i];
    return b;
}

int check_desc(const vfb_domain_desc *d)
{
    if (!d)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "domain description is NULL");
    if (d->nx < 2 || d->ny < 2 || d->nz < 2 || d->nx > 65535 || d->ny > 65535 || d->nz > 65535)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "domain extents must lie in [2, 65535]");
    if ((uint64_t)d->nx * d->ny * d->nz >= (1ull << 31))
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "domain has too many nodes");
    if (!(d->omega > 0.0 && d->omega < 2.0))
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "omega must lie in (0, 2)");
    return VFB_OK;
}

bool needs_mask(const vfb_domain_desc *d, bool user_mask)
{
    return user_mask || !d->periodic_x || !d->periodic_y || !d->periodic_z;
}

void domain_sizes(const vfb_pool *p, const vfb_domain_desc *d, bool has_mask, uint64_t &pitch, uint64_t &pop_bytes,
                  uint64_t &mask_bytes)
{
    const uint64_t n = (uint64_t)d->nx * d->ny * d->nz;
    const uint64_t sb = storage_size(p->desc.storage);
    const uint64_t align_el = kAlign / sb;
    pitch = (n + align_el - 1) / align_el * align_el;
    pop_bytes = 27 * pitch * sb;
    mask_bytes = has_mask ? align_up(n) : 0;
}

// arena bytes of a domain's BC lists: no-slip k, cut masks with the first link of every 32 nodes,
// the q of the cut links, guard tables and saved values; pressure k, kN, direction and drho
struct BCSizes {
    uint64_t noslip_k, noslip_cut, noslip_q, noslip_guard, noslip_saved, pressure_i, pressure_rho;
    uint64_t total() const
    {
        return noslip_k + noslip_cut + noslip_q + noslip_guard + noslip_saved + pressure_i + pressure_rho;
    }
};

BCSizes bc_sizes(const vfb_pool *p, uint32_t n_noslip, uint64_t n_links, uint32_t n_guarded, uint32_t n_saved,
                 uint32_t n_pressure)
{
    const uint64_t rs = real_size(p->desc.storage);
    BCSizes b;
    b.noslip_k = n_noslip ? align_up(4ull * n_noslip) : 0;
    b.noslip_cut = n_noslip ? align_up(4ull * n_noslip + 4ull * ((n_noslip + 31) / 32)) : 0;
    b.noslip_q = n_links ? align_up(n_links * rs) : 0;
    b.noslip_guard = n_noslip ? align_up(8ull * n_noslip + 4ull * n_guarded) : 0;
    b.noslip_saved = n_saved ? align_up((uint64_t)n_saved * rs) : 0;
    b.pressure_i = n_pressure ? align_up(12ull * n_pressure) : 0;
    b.pressure_rho = n_pressure ? align_up((uint64_t)n_pressure * rs) : 0;
    return b;
}

// the guard tables of a domain's no-slip list (guards.h), with q tested in the pool's real type, and
// the list positions of its guarded nodes (the guard kernel's work)
uint32_t guard_tables(const vfb_pool *p, const vfb_domain_desc *d, const vfb_domain_bcs *b,
                      std::vector<uint32_t> &mask, std::vector<uint32_t> &first, std::vector<uint32_t> &guarded)
{
    const uint32_t n = b ? b->number_of_noslip_nodes : 0;
    std::vector<uint32_t> table;
    const int periodic = (d->periodic_x ? 1 : 0) | (d->periodic_y ? 2 : 0) | (d->periodic_z ? 4 : 0);
    uint32_t saved = 0;
    if (n && real_size(p->desc.storage) == 8) {
        saved = vfb::bc_guard_tables(b->noslip_k, b->noslip_q27, n, d->nx, d->ny, d->nz, periodic, table);
    } else if (n) {
        const std::vector<float> q(b->noslip_q27, b->noslip_q27 + 27ull * n);
        saved = vfb::bc_guard_tables(b->noslip_k, q.data(), n, d->nx, d->ny, d->nz, periodic, table);
    }
    mask.assign(table.begin(), table.begin() + n);
    first.assign(table.begin() + n, table.end());
    guarded.clear();
    for (uint32_t i = 0; i < n; ++i)
        if (mask[i])
            guarded.push_back(i);
    return saved;
}

// the no-slip list in the link form of the pool's kernel (pool_tables.h)
uint64_t noslip_links(const vfb_pool *p, const vfb_domain_bcs *b, std::vector<uint32_t> *cut_first,
                      std::vector<unsigned char> *q_out)
{
    return vfb::noslip_link_tables(b ? b->noslip_q27 : nullptr, b ? b->number_of_noslip_nodes : 0,
                                   real_size(p->desc.storage) == 8, cut_first, q_out);
}

bool is_axis_direction(int32_t d) { return d >= VFB_DIR_P00 && d <= VFB_DIR_00M; }

// host-side checks of a domain's BC lists against its extents and mask (1 = fluid)
int check_bcs(const vfb_domain_bcs *b, const vfb_domain_desc *d, const std::vector<uint8_t> *mask)
{
    if (!b)
        return VFB_OK;
    const uint64_t nodes = (uint64_t)d->nx * d->ny * d->nz;
    if (b->number_of_noslip_nodes) {
        if (b->noslip_variant != VFB_NOSLIP_INTERPOLATED_COMPRESSIBLE)
            return pool_fail(VFB_ERR_UNSUPPORTED, "pools run NoSlipInterpolatedCompressible no-slip lists");
        if (!b->noslip_k || !b->noslip_q27)
            return pool_fail(VFB_ERR_INVALID_ARGUMENT, "no-slip arrays are NULL");
    }
    if (b->number_of_pressure_nodes) {
        if (b->pressure_variant != VFB_PRESSURE_NON_EQUILIBRIUM_COMPRESSIBLE)
            return pool_fail(VFB_ERR_UNSUPPORTED, "pools run PressureNonEquilibriumCompressible pressure lists");
        if (!b->pressure_k || !b->pressure_k_neighbor || !b->pressure_rho || !b->pressure_direction)
            return pool_fail(VFB_ERR_INVALID_ARGUMENT, "pressure arrays are NULL");
    }
    auto fluid = [&](int32_t k) {
        return k >= 0 && (uint64_t)k < nodes && (!mask || (*mask)[(size_t)k] != 0);
    };
    for (uint32_t i = 0; i < b->number_of_noslip_nodes; ++i)
        if (!fluid(b->noslip_k[i]))
            return pool_fail(VFB_ERR_INVALID_ARGUMENT, "a no-slip BC node is outside the domain or not fluid");
    for (uint32_t i = 0; i < b->number_of_pressure_nodes; ++i) {
        if (!fluid(b->pressure_k[i]) || b->pressure_k_neighbor[i] < 0 || (uint64_t)b->pressure_k_neighbor[i] >= nodes)
            return pool_fail(VFB_ERR_INVALID_ARGUMENT, "a pressure BC node or its neighbour is outside the domain");
        if (!is_axis_direction(b->pressure_direction[i]))
            return pool_fail(VFB_ERR_INVALID_ARGUMENT, "pressure directions are VFB_DIR_P00 ... VFB_DIR_00M");
    }
    return VFB_OK;
}

} // namespace

extern "C" {

int vfb_pool_create(const vfb_pool_desc *desc, vfb_pool **out)
{
    if (!desc || !out)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    PoolOps ops;
    if (!select_ops(desc->storage, desc->arith, ops))
        return pool_fail(desc->arith == VFB_ARITH_EXACT ? VFB_ERR_UNSUPPORTED : VFB_ERR_INVALID_ARGUMENT,
                         "unknown storage, or exact arithmetic with 16-bit storage");
    if (desc->arena_bytes < kAlign || desc->max_domains == 0 || desc->max_domains > (1u << 20))
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "arena_bytes must be >= 256 and max_domains in [1, 2^20]");
    vfb_pool *p = new vfb_pool();
    p->desc = *desc;
    p->desc.arena_bytes = desc->arena_bytes / kAlign * kAlign;
    p->ops = ops;
    p->record_bytes = ops.domain_bytes();
    p->alloc = ArenaAllocator(p->desc.arena_bytes);
    p->slots.resize(desc->max_domains);
    cudaError_t e = cudaMalloc(&p->arena, p->desc.arena_bytes);
    if (e == cudaSuccess)
        e = cudaMalloc(&p->domain_table, p->record_bytes * desc->max_domains);
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&p->n_items, sizeof(uint32_t));
    if (e == cudaSuccess)
        e = cudaMemset(p->n_items, 0, sizeof(uint32_t));
    if (e == cudaSuccess)
        e = update_grid(p);
    if (e != cudaSuccess) {
        const int st = pool_cuda(e, "pool allocation");
        vfb_pool_destroy(p);
        return st;
    }
    *out = p;
    return VFB_OK;
}

int vfb_pool_destroy(vfb_pool *p)
{
    if (!p)
        return VFB_OK;
    drop_graph(p);
    cudaFree(p->arena);
    cudaFree(p->domain_table);
    cudaFree(p->items);
    cudaFree(p->n_items);
    cudaFree(p->staging);
    cudaFree(p->mass_partials);
    for (DeviceList *L : { &p->noslip_list, &p->guard_list, &p->pressure_list }) {
        cudaFree(L->items);
        cudaFree(L->count);
    }
    delete p;
    return VFB_OK;
}

int vfb_pool_domain_bytes(const vfb_pool *p, const vfb_domain_desc *d, int32_t has_mask, uint64_t *bytes)
{
    return vfb_pool_domain_bytes_with_bcs(p, d, has_mask, nullptr, bytes);
}

int vfb_pool_domain_bytes_with_bcs(const vfb_pool *p, const vfb_domain_desc *d, int32_t has_mask,
                                   const vfb_domain_bcs *bcs, uint64_t *bytes)
{
    if (!p || !bytes)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    int st = check_desc(d);
    if (st)
        return st;
    st = check_bcs(bcs, d, nullptr);
    if (st)
        return st;
    uint64_t pitch, pop, mask;
    domain_sizes(p, d, needs_mask(d, has_mask != 0), pitch, pop, mask);
    std::vector<uint32_t> gm, gf, gi;
    const uint32_t n_saved = guard_tables(p, d, bcs, gm, gf, gi);
    *bytes = pop + mask + bc_sizes(p, bcs ? bcs->number_of_noslip_nodes : 0, noslip_links(p, bcs, nullptr, nullptr),
                                   (uint32_t)gi.size(), n_saved, bcs ? bcs->number_of_pressure_nodes : 0).total();
    return VFB_OK;
}

int vfb_pool_add_domain(vfb_pool *p, const vfb_domain_desc *d, const uint8_t *user_mask, uint32_t *id)
{
    return vfb_pool_add_domain_with_bcs(p, d, user_mask, nullptr, id);
}

namespace {
// host array of the pool's real type from doubles
std::vector<unsigned char> to_real(const vfb_pool *p, const double *v, size_t n)
{
    const size_t rs = real_size(p->desc.storage);
    std::vector<unsigned char> out(n * rs);
    if (rs == 8) {
        std::memcpy(out.data(), v, n * 8);
    } else {
        for (size_t i = 0; i < n; ++i) {
            const float f = (float)v[i];
            std::memcpy(out.data() + 4 * i, &f, 4);
        }
    }
    return out;
}
} // namespace

int vfb_pool_add_domain_with_bcs(vfb_pool *p, const vfb_domain_desc *d, const uint8_t *user_mask,
                                 const vfb_domain_bcs *bcs, uint32_t *id)
{
    if (!p || !id)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    int st = check_desc(d);
    if (st)
        return st;
    uint32_t slot = 0;
    while (slot < p->slots.size() && (p->slots[slot].live || p->slots[slot].retired))
        ++slot;
    if (slot == p->slots.size())
        return pool_fail(VFB_ERR_OUT_OF_MEMORY, "the pool holds max_domains domains already");
    DomainSlot ds;
    ds.desc = *d;
    ds.nodes = (uint64_t)d->nx * d->ny * d->nz;
    ds.has_mask = needs_mask(d, user_mask != nullptr);
    std::vector<uint8_t> m;
    if (ds.has_mask) {
        // walls of the non-periodic axes, then the caller's solid nodes
        m.assign(ds.nodes, 1);
        const int nx = d->nx, ny = d->ny, nz = d->nz;
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    const uint64_t k = (uint64_t)x + (uint64_t)nx * ((uint64_t)y + (uint64_t)ny * z);
                    const bool wall = (!d->periodic_x && (x == 0 || x == nx - 1)) ||
                                      (!d->periodic_y && (y == 0 || y == ny - 1)) ||
                                      (!d->periodic_z && (z == 0 || z == nz - 1));
                    if (wall || (user_mask && user_mask[k] == 0))
                        m[k] = 0;
                }
    }
    st = check_bcs(bcs, d, ds.has_mask ? &m : nullptr);
    if (st)
        return st;
    ds.n_noslip = bcs ? bcs->number_of_noslip_nodes : 0;
    ds.n_pressure = bcs ? bcs->number_of_pressure_nodes : 0;
    std::vector<uint32_t> guard_mask, guard_first, guarded;
    const uint32_t n_saved = guard_tables(p, d, bcs, guard_mask, guard_first, guarded);
    ds.n_guarded = (uint32_t)guarded.size();
    uint64_t pop, mask;
    domain_sizes(p, d, ds.has_mask, ds.pitch, pop, mask);
    std::vector<uint32_t> cut_first;
    std::vector<unsigned char> link_q;
    const uint64_t n_links = noslip_links(p, bcs, &cut_first, &link_q);
    const BCSizes bs = bc_sizes(p, ds.n_noslip, n_links, ds.n_guarded, n_saved, ds.n_pressure);
    uint64_t off = 0;
    if (!p->alloc.take(pop + mask + bs.total(), off))
        return pool_fail(VFB_ERR_OUT_OF_MEMORY, "the pool's arena has no room for this domain");
    ds.dist_offset = off;
    ds.mask_offset = off + pop;
    ds.bytes = pop + mask + bs.total();
    ds.live = true;
    vfb::PoolDomainSpec spec{};
    spec.noslip_offset = off + pop + mask;
    spec.noslip_cut_offset = spec.noslip_offset + bs.noslip_k;
    spec.noslip_q_offset = spec.noslip_cut_offset + bs.noslip_cut;
    spec.noslip_guard_offset = spec.noslip_q_offset + bs.noslip_q;
    spec.noslip_saved_offset = spec.noslip_guard_offset + bs.noslip_guard;
    spec.pressure_offset = spec.noslip_saved_offset + bs.noslip_saved;
    spec.pressure_rho_offset = spec.pressure_offset + bs.pressure_i;
    char *arena = static_cast<char *>(p->arena);
    cudaError_t e = cudaSuccess;
    if (ds.has_mask)
        e = cudaMemcpy(arena + ds.mask_offset, m.data(), ds.nodes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && ds.n_noslip) {
        e = cudaMemcpy(arena + spec.noslip_offset, bcs->noslip_k, 4ull * ds.n_noslip, cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(arena + spec.noslip_cut_offset, cut_first.data(), 4ull * cut_first.size(),
                           cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !link_q.empty())
            e = cudaMemcpy(arena + spec.noslip_q_offset, link_q.data(), link_q.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(arena + spec.noslip_guard_offset, guard_mask.data(), 4ull * ds.n_noslip,
                           cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(arena + spec.noslip_guard_offset + 4ull * ds.n_noslip, guard_first.data(),
                           4ull * ds.n_noslip, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && ds.n_guarded)
            e = cudaMemcpy(arena + spec.noslip_guard_offset + 8ull * ds.n_noslip, guarded.data(),
                           4ull * ds.n_guarded, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess && ds.n_pressure) {
        const uint64_t n4 = 4ull * ds.n_pressure;
        e = cudaMemcpy(arena + spec.pressure_offset, bcs->pressure_k, n4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(arena + spec.pressure_offset + n4, bcs->pressure_k_neighbor, n4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(arena + spec.pressure_offset + 2 * n4, bcs->pressure_direction, n4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            const auto r = to_real(p, bcs->pressure_rho, ds.n_pressure);
            e = cudaMemcpy(arena + spec.pressure_rho_offset, r.data(), r.size(), cudaMemcpyHostToDevice);
        }
    }
    std::vector<unsigned char> rec(p->record_bytes);
    const uint64_t sb = storage_size(p->desc.storage);
    spec.dist_offset = ds.dist_offset / sb;
    spec.pitch = ds.pitch;
    spec.mask_offset = ds.mask_offset;
    spec.nx = d->nx;
    spec.ny = d->ny;
    spec.nz = d->nz;
    spec.flags = (d->periodic_x ? 1 : 0) | (d->periodic_y ? 2 : 0) | (d->periodic_z ? 4 : 0) | (ds.has_mask ? 8 : 0) |
                 (ds.has_mask && vfb::compact_collision(m) ? 16 : 0);
    spec.omega = d->omega;
    for (int i = 0; i < 3; ++i) {
        spec.lim[i] = d->quadric_limiters[i];
        spec.half_force[i] = d->forces[i] * 0.5;
    }
    spec.n_noslip = ds.n_noslip;
    spec.n_guarded = ds.n_guarded;
    spec.n_pressure = ds.n_pressure;
    p->ops.domain(rec.data(), spec);
    if (e == cudaSuccess)
        e = cudaMemcpy(static_cast<char *>(p->domain_table) + (size_t)slot * p->record_bytes, rec.data(), p->record_bytes,
                       cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        p->alloc.give(ds.dist_offset, ds.bytes);
        return pool_cuda(e, "pool add domain");
    }
    p->slots[slot] = ds;
    *id = slot;
    return VFB_OK;
}

int vfb_pool_remove_domain(vfb_pool *p, uint32_t id)
{
    if (!p || id >= p->slots.size() || !p->slots[id].live)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "no such domain");
    DomainSlot &d = p->slots[id];
    // steps already queued may still read the domain: its range and slot are retired now and
    // become reusable once the pool's stream has drained (vfb_pool_synchronize, or the next step)
    if (d.active)
        p->list_dirty = true;
    d.live = false;
    d.active = false;
    d.retired = true;
    return VFB_OK;
}

int vfb_pool_synchronize(vfb_pool *p, void *stream)
{
    if (!p)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "NULL pool");
    cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    if (e == cudaSuccess)
        reclaim(p);
    return pool_cuda(e, "pool synchronize");
}

int vfb_pool_init_domain(vfb_pool *p, uint32_t id, const void *rho, const void *ux, const void *uy, const void *uz,
                         int32_t from_host, void *stream)
{
    if (!p || id >= p->slots.size() || !p->slots[id].live)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "no such domain");
    if (!rho || !ux || !uy || !uz)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "NULL field");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DomainSlot &d = p->slots[id];
    const uint64_t fb = d.nodes * real_size(p->desc.storage);
    const void *dev[4] = { rho, ux, uy, uz };
    cudaError_t e = cudaSuccess;
    if (from_host) {
        e = ensure_staging(p, 4 * fb, s);
        const void *src[4] = { rho, ux, uy, uz };
        for (int i = 0; i < 4 && e == cudaSuccess; ++i) {
            void *dst = static_cast<char *>(p->staging) + i * fb;
            e = cudaMemcpyAsync(dst, src[i], fb, cudaMemcpyHostToDevice, s);
            dev[i] = dst;
        }
    }
    // PreProcessorImp::init writes the odd, then the even parity; here the pool's current parity
    // is written last, so the domain joins the shared step sequence wherever it stands
    const vfb::BoxState b = domain_box(p, d);
    if (e == cudaSuccess)
        e = p->ops.init(b, !p->even, dev[0], dev[1], dev[2], dev[3], s);
    if (e == cudaSuccess)
        e = p->ops.init(b, p->even, dev[0], dev[1], dev[2], dev[3], s);
    if (from_host && e == cudaSuccess)
        e = cudaStreamSynchronize(s);   // the host arrays may be released when the call returns
    if (e == cudaSuccess && !d.active) {
        d.active = true;
        p->list_dirty = true;
    }
    d.has_ref = false;
    return pool_cuda(e, "pool init domain");
}

int vfb_pool_step(vfb_pool *p, uint32_t steps, void *stream)
{
    if (!p)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "NULL pool");
    const vfb::NvtxRange range("vfb_pool_step");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaSuccess;
    if (p->list_dirty)
        e = rebuild_list(p, s);
    uint32_t done = 0;
    const bool graphs = p->use_graph && s != nullptr;
    while (e == cudaSuccess && done < steps) {
        if (graphs && p->even && steps - done >= kGraphSteps) {
            e = ensure_graph(p, s);
            if (e == cudaSuccess)
                e = cudaGraphLaunch(p->graph, s);
            p->launches += (uint64_t)kGraphSteps * launches_per_step(p);
            done += kGraphSteps;   // an even number of steps: the parity is unchanged
            continue;
        }
        e = launch_step(p, p->even, s);
        p->even = !p->even;
        ++done;
    }
    return pool_cuda(e, "pool step");
}

int vfb_pool_domain_fields(vfb_pool *p, uint32_t id, void *rho, void *ux, void *uy, void *uz, int32_t to_host,
                           void *stream)
{
    if (!p || id >= p->slots.size() || !p->slots[id].live)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "no such domain");
    if (!rho || !ux || !uy || !uz)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "NULL field");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DomainSlot &d = p->slots[id];
    const uint64_t fb = d.nodes * real_size(p->desc.storage);
    void *out[4] = { rho, ux, uy, uz };
    void *dev[4] = { rho, ux, uy, uz };
    cudaError_t e = cudaSuccess;
    if (to_host) {
        e = ensure_staging(p, 4 * fb, s);
        for (int i = 0; i < 4; ++i)
            dev[i] = static_cast<char *>(p->staging) + i * fb;
    }
    if (e == cudaSuccess)
        e = p->ops.macros(domain_box(p, d), p->even, dev[0], dev[1], dev[2], dev[3], s);
    for (int i = 0; i < 4 && e == cudaSuccess && to_host; ++i)
        e = cudaMemcpyAsync(out[i], dev[i], fb, cudaMemcpyDeviceToHost, s);
    if (to_host && e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    return pool_cuda(e, "pool domain fields");
}

int vfb_pool_set_launch(vfb_pool *p, int32_t threads, int32_t nodes_per_thread, int32_t blocks_per_sm, int32_t use_graph)
{
    if (!p)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "NULL pool");
    if (threads != 64 && threads != 128 && threads != 256)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "threads_per_block must be 64, 128 or 256");
    if (nodes_per_thread < 1 || nodes_per_thread > 32 || blocks_per_sm < -1 || blocks_per_sm > 32)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "nodes_per_thread must lie in [1, 32], blocks_per_sm in [-1, 32]");
    if (threads != p->threads || nodes_per_thread != p->nodes_per_thread) {
        p->list_dirty = true;
        drop_graph(p);
    }
    p->threads = threads;
    p->nodes_per_thread = nodes_per_thread;
    p->blocks_per_sm = blocks_per_sm;
    p->use_graph = use_graph ? 1 : 0;
    return pool_cuda(update_grid(p), "pool launch shape");
}

int vfb_pool_get_launch(const vfb_pool *p, int32_t out4[4])
{
    if (!p || !out4)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    out4[0] = p->threads;
    out4[1] = p->nodes_per_thread;
    out4[2] = p->blocks_per_sm < 0 ? -1 : (int32_t)(p->grid / (unsigned)sm_count_here());
    out4[3] = p->use_graph;
    return VFB_OK;
}

int vfb_pool_autotune(vfb_pool *p, uint32_t trial_steps, void *stream, double *best_ms)
{
    if (!p || trial_steps == 0)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "NULL pool or no trial steps");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    struct Shape { int t, npt, bps; };
    static const Shape kShapes[] = { { 128, 1, 0 }, { 128, 2, 0 }, { 128, 4, 0 }, { 64, 1, 0 }, { 64, 2, 0 },
                                     { 256, 1, 0 }, { 256, 2, 0 }, { 128, 1, 2 }, { 128, 2, 2 },
                                     { 128, 4, -1 }, { 128, 8, -1 }, { 256, 4, -1 }, { 64, 8, -1 },
                                     { 128, 16, -1 }, { 64, 16, -1 } };
    const int graph = p->use_graph;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaEventCreate(&a);
    if (e == cudaSuccess)
        e = cudaEventCreate(&b);
    double best = 1e300;
    Shape pick = { p->threads, p->nodes_per_thread, p->blocks_per_sm };
    for (const Shape &sh : kShapes) {
        if (e != cudaSuccess)
            break;
        int st = vfb_pool_set_launch(p, sh.t, sh.npt, sh.bps, 0);
        if (st)
            break;
        st = vfb_pool_step(p, 2, stream);
        if (st)
            break;
        e = cudaEventRecord(a, s);
        if (e == cudaSuccess)
            st = vfb_pool_step(p, trial_steps, stream);
        if (st)
            break;
        e = cudaEventRecord(b, s);
        if (e == cudaSuccess)
            e = cudaEventSynchronize(b);
        float ms = 0.f;
        if (e == cudaSuccess)
            e = cudaEventElapsedTime(&ms, a, b);
        const double per = (double)ms / trial_steps;
        if (e == cudaSuccess && per < best) {
            best = per;
            pick = sh;
        }
    }
    if (a)
        cudaEventDestroy(a);
    if (b)
        cudaEventDestroy(b);
    if (e != cudaSuccess)
        return pool_cuda(e, "pool autotune");
    if (best_ms)
        *best_ms = best;
    return vfb_pool_set_launch(p, pick.t, pick.npt, pick.bps, graph);
}

int vfb_pool_stats(const vfb_pool *p, uint32_t *active_domains, uint64_t *active_nodes, uint64_t *used_bytes,
                   uint64_t *free_bytes)
{
    if (!p)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "NULL pool");
    uint32_t n = 0;
    uint64_t nodes = 0;
    for (const DomainSlot &d : p->slots)
        if (d.live && d.active) {
            ++n;
            nodes += d.nodes;
        }
    if (active_domains)
        *active_domains = n;
    if (active_nodes)
        *active_nodes = nodes;
    if (used_bytes)
        *used_bytes = p->alloc.used();
    if (free_bytes)
        *free_bytes = p->desc.arena_bytes - p->alloc.used();
    return VFB_OK;
}

int vfb_pool_domain_mass(vfb_pool *p, double *mass, void *stream)
{
    if (!p || !mass)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaSuccess;
    if (p->list_dirty)
        e = rebuild_list(p, s);
    const size_t n = p->host_items.size();
    if (e == cudaSuccess && n > p->mass_capacity) {
        e = cudaStreamSynchronize(s);
        if (e == cudaSuccess) {
            cudaFree(p->mass_partials);
            p->mass_partials = nullptr;
            p->mass_capacity = 0;
            e = cudaMalloc((void **)&p->mass_partials, n * sizeof(double));
            if (e == cudaSuccess)
                p->mass_capacity = n;
        }
    }
    if (e == cudaSuccess)
        e = p->ops.mass(p->arena, p->domain_table, p->items, (uint32_t)n, p->nodes_per_thread, p->threads, p->even,
                        p->mass_partials, s);
    std::vector<double> partial(n);
    if (e == cudaSuccess && n)
        e = cudaMemcpyAsync(partial.data(), p->mass_partials, n * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return pool_cuda(e, "pool domain mass");
    ++p->launches;
    for (size_t i = 0; i < p->slots.size(); ++i)
        mass[i] = 0.0;
    // items are grouped by domain in id order: a fixed summation order per domain
    for (size_t i = 0; i < n; ++i)
        mass[p->host_items[i].x] += partial[i];
    return VFB_OK;
}

int vfb_pool_watchdog(vfb_pool *p, double max_relative_drift, uint32_t *failed, uint32_t capacity, uint32_t *n_failed,
                      void *stream)
{
    if (!p || !n_failed || (capacity && !failed) || !(max_relative_drift > 0.0))
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument or non-positive drift bound");
    std::vector<double> mass(p->slots.size());
    int st = vfb_pool_domain_mass(p, mass.data(), stream);
    if (st)
        return st;
    uint32_t bad = 0;
    for (uint32_t id = 0; id < p->slots.size(); ++id) {
        DomainSlot &d = p->slots[id];
        if (!d.live || !d.active)
            continue;
        const double m = mass[id];
        bool ok = std::isfinite(m);
        if (ok && !d.has_ref) {
            d.ref_mass = m;
            d.has_ref = true;
        } else if (ok) {
            ok = std::fabs(m - d.ref_mass) <= max_relative_drift * std::fabs(d.ref_mass);
        }
        if (!ok) {
            if (bad < capacity)
                failed[bad] = id;
            ++bad;
        }
    }
    *n_failed = bad;
    if (bad)
        return pool_fail(VFB_ERR_WATCHDOG, "non-finite populations or mass drift in a pool domain");
    return VFB_OK;
}

int vfb_pool_kernel_launches(const vfb_pool *p, uint64_t *count)
{
    if (!p || !count)
        return pool_fail(VFB_ERR_INVALID_ARGUMENT, "NULL argument");
    *count = p->launches;
    return VFB_OK;
}

} // extern "C"
