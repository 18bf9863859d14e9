// GPU entry points of the engine: engine_cuda_load (src/runner_cuda.cu:2931-3545) and
// engine_nonbond_cuda (src/runner_cuda.cu:2287-2628), plus device selection, the
// device-resident evaluation used to time the kernels alone, CUDA-graph replay, the launch
// autotuner and batches of independent engines (replicas) evaluated by one launch.
//
// Per evaluation: pack the cells' particles (cell-relative float positions + type, id)
// into pinned host buffers, one host->device copy each, zero the fixed-point force and
// energy accumulators, sort_cells, sweep, one device->host copy of forces and per-cell
// energies, unpack into the cells.  All launches go to one stream; CUDA events around the
// kernels give the device time.
//
// One device state (NbState) serves a list of engines: a single engine (engine_cuda_load)
// or a batch of replicas (engine_batch_create).  The engines' cells are concatenated
// (engine k's cell c is global cell cell_off[k] + c), their particle ids offset by
// id_off[k], and their tasks concatenated into one task list and one queue; each task
// carries its own sort-distance bound and shift norm and each cell its own sort scale, so
// replicas may have different boxes and cell sizes.  They must share the potential tables,
// the cutoff and the flags.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include <atomic>
#include <cstdint>
#if defined(__x86_64__)
#include <immintrin.h>
#endif
#include <utility>
#include <cmath>
#include <ctime>
#include <cuda_runtime.h>
#include "mdcore_b200.h"
#include "internal.h"
#include "nb_tuned.cuh"
#include "nb_resident.cuh"
#include "host_pool.h"

using namespace nb;

namespace {

struct NbState {
    int device = 0;
    cudaStream_t stream = nullptr;         // launch stream (own_stream unless the caller set one)
    cudaStream_t own_stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;       // around sort + sweep
    cudaEvent_t evs0 = nullptr, evs1 = nullptr;     // around the sweep kernel alone
    // engines served by this state and their offsets in the global cell / id numbering
    std::vector<struct engine*> engines;
    std::vector<int> cell_off, id_off;
    std::vector<struct cell*> flat_cells;  // every engine's cells in global order
    std::vector<cudaEvent_t> chunk_ev;     // one per download chunk
    struct nb_stats bstats = {};           // totals of the last evaluation over all engines
    // geometry
    int ncells = 0, ntasks = 0, ncap = 0, nid = 0;
    float bias = 0.f, dscale = 0.f;        // of engine 0 (used by the no-alloc entry point)
    int dmaxdist = 0;
    int maxcount = 0;
    float cut2p = 0.f, cut2s = 0.f;        // pair and self cutoff^2 (src/runner_dopair.c:577, 896)
    int unsorted = 0;
    // tables
    int npots = 0, ncoef = 0, max_type = 0;
    // tuning
    int warps = 4;
    int window = 4;                // sweep steps per register reduce-scatter (4 or 8)
    int layout = 0;                // persistent sweep: 0 = 32 i per warp, 1 = 8 i x 4 j tile
    int stages = 1;                // staging buffers per worker warp (2: next task's copies in flight)
    int occupancy = 640;           // resident threads per SM the sweep's registers are sized for
    bool has_excl = false;
    bool need_pid = false;         // ids uploaded: exclusions or explicit charges
    int ep_pot = -1;               // table index of the explicit electrostatic potential
    int tab_global = 0;            // tables read from global memory (too large for shared)
    float* d_qid = nullptr;        // charges by global id (explicit electrostatics)
    std::vector<float> h_qid;
    bool one_pot = false;           // every type pair uses table 0 (no per-pair lookup)
    int plain = 0;                 // 1: one CTA per task (the plain form); 0: persistent queue
    int fp32acc = 0;               // plain form: forces accumulated in FP32 (float atomics)
    float* d_force32 = nullptr;    // float forces of FP32 accumulation (3 per slot)
    size_t force32_slots = 0;
    // Resident steps: steepest-descent update instead of the time step (sd_gamma > 0), and a
    // per-step energy log (elog_cap records, 0 = off).
    float sd_gamma = 0.f, sd_dmax = 0.f;
    int elog_cap = 0;
    unsigned long long* r_elog = nullptr;    // elog_cap x {step number, epot, ekin, 0}
    unsigned long long* r_eacc = nullptr;    // the step's kinetic-energy accumulator, step-number base
    // Verlet skin of the resident steps (engine_flag_verlet): rebuild flag and counters,
    // reference positions by slot, per-cell displacement in key units.
    bool verlet = false;
    float verlet_skin = 0.f;
    int* r_vw = nullptr;
    float4* r_oldx = nullptr;
    int* r_cell_mdx = nullptr;
    int* d_order = nullptr;        // task queue order (scheduling order of all tasks)
    int* d_queue = nullptr;        // compacted queue of the current step
    int* d_qcount = nullptr;
    int* d_bsum = nullptr;
    bool compact = false;          // rebuild the queue each step without empty tasks
    int* d_counter = nullptr;      // queue head
    long long* d_task_clock = nullptr;
    int* d_task_sm = nullptr;
    int record_clock = 0;
    int sm_count = 0;
    // CUDA graph of one evaluation's launches (memsets, sort, queue, sweep)
    bool use_graph = false;
    bool capturing = false;
    int last_grid = 0;             // grid of the last direct persistent launch
    int buf_gen = 0;               // bumped whenever device buffers move
    long long graph_key = -1, prepared_key = -1;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    // device buffers
    float4* d_xq = nullptr;
    int* d_pid = nullptr;
    unsigned* d_keys = nullptr;
    unsigned long long* d_force = nullptr;
    int* d_cstart = nullptr;
    int* d_ccount = nullptr;
    unsigned* d_cmask = nullptr;
    float2* d_cscale = nullptr;    // per cell: sort scale 32767/(2|h|) and bias |h|
    unsigned long long* d_acc = nullptr;
    unsigned long long* d_cell_epot = nullptr;   // 2 * ncells: energies, then virials
    TaskRec* d_tasks = nullptr;
    float4* d_tshift = nullptr;
    float* d_coef = nullptr;
    float4* d_potinfo = nullptr;
    int* d_potn = nullptr;
    int* d_potidx = nullptr;
    unsigned* d_emask = nullptr;
    int* d_exoff = nullptr;
    int* d_exlist = nullptr;
    // pinned host buffers
    float4* h_xq = nullptr;
    int* h_pid = nullptr;
    int* h_cstart = nullptr;    // ncells+1 followed by ncells counts
    unsigned long long* h_force = nullptr;   // pinned; holds float forces (3 per slot)
    float* d_forcef = nullptr;
    unsigned long long* h_cell_epot = nullptr;   // 2 * ncells
    unsigned long long* h_acc = nullptr;
    bool resident_valid = false;
    // Device-resident steps (nb_resident.cuh): fixed blocks of capc slots per cell, two
    // sides (re-binning writes the other side), static per-id fields for the host copy.
    bool res_active = false;
    bool res_dirty = false;            // the device holds steps the host cells do not
    int capc = 0, rside = 0, mcap = 16, res_margin = 8;
    long long res_nparts = 0, res_done = 0, res_done_total = 0, res_pairs = 0, res_pairs_total = 0;
    int res_regrows = 0;
    int* r_cnt[2] = {nullptr, nullptr};      // particles per cell of each side
    unsigned long long* r_done = nullptr;    // completed resident steps, their accepted pairs
    float4* r_xq[2] = {nullptr, nullptr};
    float4* r_v[2] = {nullptr, nullptr};
    int* r_pid[2] = {nullptr, nullptr};
    int *r_cstart = nullptr, *r_nstay = nullptr, *r_nmove = nullptr, *r_slot_of = nullptr;
    int *r_nbr = nullptr, *r_cell_engine = nullptr;
    float4* r_cell_h = nullptr;
    float* r_engine_dt = nullptr;
    double* r_engine_imass = nullptr;
    Mover* r_movers = nullptr;
    unsigned* r_keys = nullptr;
    unsigned long long* r_force = nullptr;
    unsigned long long* r_status = nullptr;
    // Dense copies of the particles in cell order, 3 float4 per particle of room.  Upload:
    // position + type bits, velocity + global id bits (float4 each), and with explicit
    // electrostatics the charges from float 10 np.  Download: position + upload-index bits
    // (float4), then velocities and forces as float triples (40 bytes per particle).
    float4* r_dense = nullptr;
    float4* h_dense = nullptr;         // downloads (pinned)
    float4* h_up = nullptr;            // uploads (pinned): positions, velocities
    int *r_doff = nullptr, *h_rcount = nullptr;
    int* r_bsum = nullptr;                   // block sums of the count scan
    // Bonds of the resident steps (built with the device blocks).
    int nbonds = 0;
    long long bonds_key = -1;              // sum of the engines' bonds_gen the bonds were built from
    int4* r_bonds = nullptr;
    float* r_bcoef = nullptr;
    float4* r_bpotinfo = nullptr;
    int* r_bpotn = nullptr;
    double2* r_bab2 = nullptr;
    int* r_eng_cell0 = nullptr;
    int4* r_eng_cdim = nullptr;
    double4* r_eng_h = nullptr;
    unsigned long long* r_ebond = nullptr;   // bond, angle, dihedral energy per engine (3 x engines)
    unsigned long long* h_ebond = nullptr;
    int nangles = 0, ndihedrals = 0;
    int4* r_angles = nullptr;                // i, j, k, engine << 16 | table
    int4* r_dihedrals = nullptr;             // i, j, k, l
    int* r_dihedral_te = nullptr;            // engine << 16 | table
    double2* r_bab = nullptr;                // per table: a, b
    unsigned long long* h_words = nullptr;   // status, completed steps, their pairs (pinned)
    std::vector<long long> res_engine_n;   // particles of each engine on the device
    // What the device does not carry, and the global id, by dense index of the last upload
    // (cell order): the download returns each particle's upload index, so the host reads
    // these nearly in order instead of scattering by particle id.
    struct alignas(16) UpAux {
        int gid;
        float q;
        int vid;
        short type;
        unsigned short flags;
    };
    std::vector<UpAux> up_aux;
    int* r_up_of = nullptr;            // device: global id -> dense index of the last upload
    cudaGraph_t rgraph[2] = {nullptr, nullptr};
    cudaGraphExec_t rgraph_exec[2] = {nullptr, nullptr};
    long long rgraph_key[2] = {-1, -1}, rprepared[2] = {-1, -1};
    void* sched = nullptr;             // learned-scheduler state (SchedState)
    // engine_step of a batch in groups of engines (engine_batch_setgroups): one device state
    // and stream per group, so that the host packing and unpacking of one group overlap the
    // uploads, steps and downloads of the others.  Built at the first grouped step.
    int groups_req = 0;                // 0: automatic
    std::vector<NbState*> groups;
    int max_chunks = 8;                // pipeline chunks of one engine_step transfer
    int tiny_inherited = -1;           // a group's Params::tiny, its batch's (-1: from its own counts)
    std::vector<int> heur_order;       // count-product order built at load
};

void sched_free(void* p);

int cuda_fail(cudaError_t err, int line, const char* func) {
    errs_register(engine_err_cuda, cudaGetErrorString(err), line, func, __FILE__);
    engine_err = engine_err_cuda;
    return engine_err_cuda;
}

#define CU(call)                                                           \
    do {                                                                   \
        cudaError_t err_ = (call);                                         \
        if (err_ != cudaSuccess) return cuda_fail(err_, __LINE__, __func__); \
    } while (0)

NbState* state(struct engine* e) { return static_cast<NbState*>(e->cuda); }

// Estimated cost of a task (the reference's METIS cell-pair weights).
double task_weight(int sid, double ni, double nj) {
    if (sid < 0) return ni * ni - ni;
    const int idx = 26 - sid;                         // direction index, see sort_axis
    const int nz = (idx / 9 != 1) + ((idx / 3) % 3 != 1) + (idx % 3 != 1);
    const double w = nz == 1 ? 0.50004 : (nz == 2 ? 0.16176 : 0.036213);
    return ni * nj * w;
}

// A queue order with locality from task costs: the tasks, in the cell-major order they were
// generated in, are cut into tiles of `tile` consecutive tasks; each tile's cost is the sum
// of its tasks' costs, and the tiles go in decreasing cost class (a factor of 2^(1/4) per
// class) and, within a class, in cell-major order, each tile's tasks by decreasing cost.
std::vector<int> tiled_order(const std::vector<double>& cost, int n, int tile) {
    const int ntiles = (n + tile - 1) / tile;
    std::vector<double> tcost(ntiles, 0.0);
    for (int t = 0; t < n; t++) tcost[t / tile] += std::max(0.0, cost[t]);
    std::vector<int> cls(ntiles);
    for (int b = 0; b < ntiles; b++)
        cls[b] = tcost[b] > 0.0 ? (int)std::floor(4.0 * std::log2(tcost[b])) : INT_MIN;
    std::vector<int> tiles(ntiles);
    for (int b = 0; b < ntiles; b++) tiles[b] = b;
    std::stable_sort(tiles.begin(), tiles.end(), [&](int a, int b) { return cls[a] > cls[b]; });
    std::vector<int> order;
    order.reserve(n);
    for (int b : tiles) {
        const int t0 = b * tile, t1 = std::min(n, t0 + tile);
        const size_t first = order.size();
        for (int t = t0; t < t1; t++) order.push_back(t);
        std::stable_sort(order.begin() + first, order.end(), [&](int a, int c) { return cost[a] > cost[c]; });
    }
    return order;
}

// Tiles of the automatic size: about an eighth of the tasks per worker warp of the
// persistent sweep (at `occupancy` threads per SM), so that every warp still takes several.
int auto_tile(int ntasks, int sm_count, int occupancy) {
    const long long workers = (long long)sm_count * (occupancy / 32);
    return (int)std::max(1LL, ntasks / std::max(1LL, 8 * workers));
}

float bits_as_float(int v) {
    float f;
    std::memcpy(&f, &v, sizeof(f));
    return f;
}

template <typename T>
int dev_alloc(T** p, size_t n) {
    CU(cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T) + 16));
    return 0;
}

// (Re)allocates the per-particle buffers for `ncap` slots.
int alloc_particles(NbState* st, int ncap) {
    if (ncap <= st->ncap) return 0;
    ncap = ncap + ncap / 8 + 64;
    cudaFree(st->d_xq); cudaFree(st->d_pid); cudaFree(st->d_keys); cudaFree(st->d_force);
    st->d_xq = nullptr; st->d_pid = nullptr; st->d_keys = nullptr; st->d_force = nullptr;
    cudaFreeHost(st->h_xq); cudaFreeHost(st->h_pid); cudaFreeHost(st->h_force);
    st->h_xq = nullptr; st->h_pid = nullptr; st->h_force = nullptr;
    ++st->buf_gen;
    if (dev_alloc(&st->d_xq, ncap) || dev_alloc(&st->d_pid, ncap) || dev_alloc(&st->d_keys, 13 * (size_t)ncap) ||
        dev_alloc(&st->d_force, 3 * (size_t)ncap))
        return engine_err_cuda;
    // Upload buffers are only written by the host: write-combined pages take the writes
    // without reading the lines first and stream faster over PCIe.
    CU(cudaMallocHost(&st->h_xq, sizeof(float4) * ncap));
    CU(cudaMallocHost(&st->h_pid, sizeof(int) * ncap));
    CU(cudaMallocHost(&st->h_force, sizeof(unsigned long long) * 3 * ncap));
    cudaFree(st->d_forcef);
    if (dev_alloc(&st->d_forcef, 3 * (size_t)ncap)) return engine_err_cuda;
    CU(cudaMemset(st->d_xq, 0, sizeof(float4) * ncap));
    CU(cudaMemset(st->d_pid, 0, sizeof(int) * ncap));
    st->ncap = ncap;
    return 0;
}

// Fixed-point forces (int64, 2^24 units) to float, for the copy back to the host.
__global__ void fixed_to_float(const unsigned long long* __restrict__ f, float* __restrict__ out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)((double)(long long)f[i] * (1.0 / (double)kForceScale));
}

// Evicts [p, p + bytes) from the host caches (writing dirty lines back).  The pinned upload
// and download buffers are written or read by many host threads; lines left in their caches
// make the copy engine snoop every core (measured: uploads of 3 MB at 6 GB/s instead of
// 50 GB/s), so each thread evicts what it has written or read.
#if defined(__x86_64__)
__attribute__((target("clflushopt"))) static void evict_lines_opt(const void* p, size_t bytes) {
    const char* c = reinterpret_cast<const char*>(reinterpret_cast<uintptr_t>(p) & ~uintptr_t(63));
    const char* e = static_cast<const char*>(p) + bytes;
    for (; c < e; c += 64) _mm_clflushopt(const_cast<char*>(c));
}
#endif

void evict_lines(const void* p, size_t bytes) {
#if defined(__x86_64__)
    static const bool opt = __builtin_cpu_supports("clflushopt");
    if (opt) {
        evict_lines_opt(p, bytes);
        return;
    }
    const char* c = reinterpret_cast<const char*>(reinterpret_cast<uintptr_t>(p) & ~uintptr_t(63));
    const char* e = static_cast<const char*>(p) + bytes;
    for (; c < e; c += 64) _mm_clflush(c);
#else
    (void)p;
    (void)bytes;
#endif
}

// Stores into the pinned upload buffers that bypass the CPU caches (non-temporal): the copy
// engine then reads the lines from memory without snooping the host threads' caches, and no
// eviction pass is needed.  fence_nt() orders a thread's streamed stores before the copy.
inline void store_nt(float4* dst, float4 v) {
#if defined(__x86_64__)
    _mm_stream_ps(reinterpret_cast<float*>(dst), _mm_set_ps(v.w, v.z, v.y, v.x));
#else
    *dst = v;
#endif
}
inline void store_nt(int* dst, int v) {
#if defined(__x86_64__)
    _mm_stream_si32(dst, v);
#else
    *dst = v;
#endif
}
inline void store_nt(float* dst, float v) {
    int bits;
    std::memcpy(&bits, &v, sizeof(int));
    store_nt(reinterpret_cast<int*>(dst), bits);
}
inline void fence_nt() {
#if defined(__x86_64__)
    _mm_sfence();
#endif
}

double now_ms() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

// Cells per sort block: kSortWarps (one per warp) when cells hold 32 particle slots or fewer
// on average (one warp sorts a small cell alone), else 1 (the block's warps share a large
// cell's directions).
int sort_cells_per_block(int slots, int ncells) { return slots <= 32 * (long long)ncells ? kSortWarps : 1; }

// Launches sort_cells for cells of up to scap particles (its shared memory sized by scap).
int launch_sort(const float4* xq, const int* cstart, const int* ccount, const unsigned* cmask, unsigned* keys,
                const float2* cscale, int ncells, int cpc, int scap, unsigned long long* acc,
                const unsigned long long* abort, bool capturing, cudaStream_t s, const int* rebuild = nullptr) {
    scap = std::max(4, std::min(kMaxPartsPerCell, (scap + 3) & ~3));
    const size_t smem = sort_smem_bytes(scap);
    // the largest size any launch asks for, so that launches captured into a graph later
    // (where the attribute is not set) are covered whatever their cells hold
    if (!capturing)
        CU(cudaFuncSetAttribute(sort_cells, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sort_smem_bytes(kMaxPartsPerCell)));
    sort_cells<<<(ncells + cpc - 1) / cpc, kSortWarps * 32, smem, s>>>(xq, cstart, ccount, cmask, keys, cscale,
                                                                       ncells, cpc, scap, acc, abort, rebuild);
    CU(cudaGetLastError());
    return 0;
}

// Particles per host-thread range of the per-step host loops (MDB_HOST_GRAIN, default
// 2,048) and per pipelined chunk of the host<->device copies (MDB_COPY_CHUNK, default
// 49,152): each chunk's copies overlap the host packing of the next one (upload) or the
// host unpacking of the previous one (download).
long long env_count(const char* name, long long dflt) {
    const char* env = std::getenv(name);
    const long long v = env ? std::atoll(env) : 0;
    return v > 0 ? v : dflt;
}
// The persistent sweeps' unstaged path for tasks of at most 32 candidate pairs (Params::tiny)
// is on for systems of fewer than 8 particles per cell on average, where such tasks are
// common (a vapour, a dilute gas); elsewhere the per-task test is left out.  A property of
// the engines' particle and cell counts, so every entry point (engine_step, resident steps,
// batches, the no-alloc call) takes the same path for the same system.
int tiny_tasks_of(const NbState* st) {
    if (st->tiny_inherited >= 0) return st->tiny_inherited;
    long long n = 0;
    for (const struct engine* e : st->engines) n += e->s.nr_parts;
    return n < 8LL * st->ncells ? 1 : 0;
}

long long host_grain_parts() {
    static const long long v = env_count("MDB_HOST_GRAIN", 2048);
    return v;
}
long long copy_chunk_parts() {
    static const long long v = env_count("MDB_COPY_CHUNK", 49152);
    return v;
}

// Cells per host-thread range: about host_grain_parts() particles, at least 16 cells.
// Cells per range of the host threads' passes over the cell records.
constexpr int kCellPassGrain = 4096;

int cell_grain(const NbState* st) {
    long long n = 0;
    for (const struct engine* e : st->engines) n += e->s.nr_parts;
    const long long avg = st->ncells > 0 ? n / st->ncells + 1 : 1;
    return (int)std::max(16LL, host_grain_parts() / avg);
}

// Slot layout of this evaluation (host threads over ranges of cells): counts, padded slot
// offsets, the largest cell; grows the buffers.  Returns the number of slots.
int prepare_slots(NbState* st) {
    HostPool& pool = HostPool::get();
    const int nc = st->ncells;
    int* cstart = st->h_cstart;
    int* ccount = st->h_cstart + nc + 1;
    const std::vector<struct cell*>& cells = st->flat_cells;
    const int parts = pool.threads();
    std::vector<int> part_slots(parts + 1, 0), part_max(parts, 0);
    const int grain = cell_grain(st);
    pool.run(nc, grain, [&](int part, int b, int e) {
        int slots = 0, maxc = 0;
        for (int c = b; c < e; c++) {
            const int n = cells[c]->count;
            ccount[c] = n;
            slots += (n + 3) & ~3;
            maxc = std::max(maxc, n);
        }
        part_slots[part + 1] = slots;
        part_max[part] = maxc;
    });
    int maxc = 0;
    for (int k = 0; k < parts; k++) {
        part_slots[k + 1] += part_slots[k];
        maxc = std::max(maxc, part_max[k]);
    }
    const int total = part_slots[parts];
    if (maxc > kMaxPartsPerCell) {
        errs_register(engine_err_maxparts, "Max. number of parts per cell exceeded.", __LINE__, __func__, __FILE__);
        return engine_err = engine_err_maxparts;
    }
    if (alloc_particles(st, total + 4) < 0) return engine_err_cuda;
    pool.run(nc, grain, [&](int part, int b, int e) {
        int slot = part_slots[part];
        for (int c = b; c < e; c++) {
            cstart[c] = slot;
            slot += (ccount[c] + 3) & ~3;
        }
    });
    cstart[nc] = total;
    st->maxcount = maxc;
    return total;
}

// Packs cells [cb, ce) into the pinned upload buffers (host threads over ranges of cells):
// positions and types, and particle ids when the system has exclusions.
void pack_range(NbState* st, int cb, int ce) {
    const int* cstart = st->h_cstart;
    HostPool::get().run(ce - cb, cell_grain(st), [&](int, int b, int e) {
        size_t k = std::upper_bound(st->cell_off.begin(), st->cell_off.end(), cb + b) - st->cell_off.begin() - 1;
        for (int c = cb + b; c < cb + e; c++) {
            while (c >= st->cell_off[k + 1]) k++;
            const int id0 = st->id_off[k];
            const struct cell* cl = st->flat_cells[c];
            const int slot = cstart[c];
            const int pad = (cl->count + 3) & ~3;
            for (int q = 0; q < cl->count; q++) {
                const struct part* p = &cl->parts[q];
                store_nt(st->h_xq + slot + q, make_float4(p->x[0], p->x[1], p->x[2], bits_as_float((int)p->type)));
            }
            for (int q = cl->count; q < pad; q++)
                store_nt(st->h_xq + slot + q, make_float4(0.f, 0.f, 0.f, bits_as_float(0)));
            if (st->need_pid) {          // ids are read by the sweep for exclusions and charges only
                for (int q = 0; q < cl->count; q++) store_nt(st->h_pid + slot + q, id0 + cl->parts[q].id);
                for (int q = cl->count; q < pad; q++) store_nt(st->h_pid + slot + q, 0);
            }
        }
        fence_nt();
    });
}

// Cell ranges of the host<->device pipeline: up to 8 chunks of about copy_chunk_parts()
// slots, so that packing (unpacking) one chunk overlaps the copy of another.
std::vector<int> chunk_bounds(const NbState* st, int total) {
    const int k = (int)std::max(1LL, std::min(8LL, total / copy_chunk_parts()));
    std::vector<int> bounds(k + 1, st->ncells);
    bounds[0] = 0;
    for (int q = 1; q < k; q++) {
        const long long target = (long long)total * q / k;
        bounds[q] = (int)(std::lower_bound(st->h_cstart, st->h_cstart + st->ncells, (int)target) - st->h_cstart);
    }
    return bounds;
}

int chunk_events(NbState* st, size_t n) {
    while (st->chunk_ev.size() < n) {
        cudaEvent_t ev;
        CU(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        st->chunk_ev.push_back(ev);
    }
    return 0;
}

template <int NW>
int launch_plain_nw(NbState* st, const Params& P, int cap, size_t smem) {
    if (!st->capturing)
        CU(cudaFuncSetAttribute(sweep_tasks<NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    sweep_tasks<NW><<<st->ntasks, NW * 32, smem, st->stream>>>(P, cap);
    CU(cudaGetLastError());
    return 0;
}

int launch_plain(NbState* st, const Params& P, int cap) {
    int nw = st->warps;
    const int tc = st->tab_global ? 0 : st->ncoef, tp = st->tab_global ? 0 : st->npots;
    size_t smem = sweep_smem_bytes(cap, nw, tc, tp, st->max_type);
    while (smem > 200 * 1024 && nw > 1) {
        nw /= 2;
        smem = sweep_smem_bytes(cap, nw, tc, tp, st->max_type);
    }
    if (smem > 220 * 1024) {
        errs_register(engine_err_maxparts, "Cell too large for the sweep kernel's shared memory.", __LINE__,
                      __func__, __FILE__);
        return engine_err = engine_err_maxparts;
    }
    switch (nw) {
        case 1: return launch_plain_nw<1>(st, P, cap, smem);
        case 2: return launch_plain_nw<2>(st, P, cap, smem);
        case 8: return launch_plain_nw<8>(st, P, cap, smem);
        default: return launch_plain_nw<4>(st, P, cap, smem);
    }
}

// Persistent launch: as many CTAs as fit on every SM at once.  Under stream capture the
// function attribute and occupancy query are skipped and the grid of the preceding direct
// launch of the same configuration is reused.
template <int NW, bool EX, int TAB, int WIN, int LAY, int STG, int TPSM, bool TINY>
int launch_tuned_k(NbState* st, const TunedParams& T, int cap, size_t smem) {
    auto kern = LAY ? sweep_tiled<NW, EX, TAB, WIN, STG, TPSM, TINY> : sweep_tuned<NW, EX, TAB, WIN, STG, TPSM, TINY>;
    int grid = st->last_grid;
    if (!st->capturing) {
        CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NW * 32, smem));
        if (per_sm < 1) per_sm = 1;
        grid = st->sm_count * per_sm;
        st->last_grid = grid;
    }
    kern<<<grid, NW * 32, smem, st->stream>>>(T, cap);
    CU(cudaGetLastError());
    return 0;
}

// The tiny-task path (Params::tiny) is compiled into the shapes of 1024 threads per SM, those
// of small cells; the other shapes, and systems that do not ask for it, run without it.
template <int NW, bool EX, int TAB, int WIN, int LAY, int STG, int TPSM>
int launch_tuned_nw(NbState* st, const TunedParams& T, int cap, size_t smem) {
    if constexpr (TPSM == 1024)
        if (T.p.tiny) return launch_tuned_k<NW, EX, TAB, WIN, LAY, STG, TPSM, true>(st, T, cap, smem);
    return launch_tuned_k<NW, EX, TAB, WIN, LAY, STG, TPSM, false>(st, T, cap, smem);
}

template <int NW, int WIN, int LAY, int STG, int TPSM>
int launch_tuned_w(NbState* st, const TunedParams& T, int cap, size_t smem) {
    if (st->tab_global)
        return st->has_excl ? launch_tuned_nw<NW, true, kTabGlobal, WIN, LAY, STG, TPSM>(st, T, cap, smem)
                            : launch_tuned_nw<NW, false, kTabGlobal, WIN, LAY, STG, TPSM>(st, T, cap, smem);
    const bool one = st->one_pot;
    if (st->has_excl)
        return one ? launch_tuned_nw<NW, true, kTabOne, WIN, LAY, STG, TPSM>(st, T, cap, smem)
                   : launch_tuned_nw<NW, true, kTabShared, WIN, LAY, STG, TPSM>(st, T, cap, smem);
    return one ? launch_tuned_nw<NW, false, kTabOne, WIN, LAY, STG, TPSM>(st, T, cap, smem)
               : launch_tuned_nw<NW, false, kTabShared, WIN, LAY, STG, TPSM>(st, T, cap, smem);
}

// Worker warps per block: 2, 4 or 8 (two warps fit even the largest cells).
template <int WIN, int LAY, int STG, int TPSM>
int launch_tuned_win(NbState* st, const TunedParams& T, int cap, size_t smem, int nw) {
    switch (nw) {
        case 2: return launch_tuned_w<2, WIN, LAY, STG, TPSM>(st, T, cap, smem);
        case 8: return launch_tuned_w<8, WIN, LAY, STG, TPSM>(st, T, cap, smem);
        default: return launch_tuned_w<4, WIN, LAY, STG, TPSM>(st, T, cap, smem);
    }
}

// Instantiated shapes: at 640 threads per SM every window and staging choice; at 768 the
// 4-step window with one staging buffer; at 1024 (small cells) one or two buffers.
template <int LAY>
int launch_tuned_lay(NbState* st, const TunedParams& T, int cap, size_t smem, int nw) {
    if (st->occupancy == 1024)
        return st->stages == 2 ? launch_tuned_win<4, LAY, 2, 1024>(st, T, cap, smem, nw)
                               : launch_tuned_win<4, LAY, 1, 1024>(st, T, cap, smem, nw);
    if (st->occupancy == 768) return launch_tuned_win<4, LAY, 1, 768>(st, T, cap, smem, nw);
    if (st->stages == 2) return launch_tuned_win<4, LAY, 2, 640>(st, T, cap, smem, nw);
    if (st->window == 8) return launch_tuned_win<8, LAY, 1, 640>(st, T, cap, smem, nw);
    return launch_tuned_win<4, LAY, 1, 640>(st, T, cap, smem, nw);
}

int launch_tuned(NbState* st, const Params& P, int cap4) {
    const int cap = cap4 + 8;
    TunedParams T;
    T.p = P;
    T.order = st->d_order;
    T.qcount = nullptr;
    if (st->compact && st->ntasks > 0) {
        const int nb = (st->ntasks + kQueueBlock - 1) / kQueueBlock;
        queue_count<<<nb, kQueueBlock, 0, st->stream>>>(st->d_order, st->d_tasks, P.ccount, st->ntasks, st->d_bsum);
        queue_offsets<<<1, kQueueBlock, 0, st->stream>>>(st->d_bsum, nb, st->d_qcount);
        queue_scatter<<<nb, kQueueBlock, 0, st->stream>>>(st->d_order, st->d_tasks, P.ccount, st->ntasks, st->d_bsum,
                                                          st->d_queue);
        CU(cudaGetLastError());
        T.order = st->d_queue;
        T.qcount = st->d_qcount;
    }
    T.counter = st->d_counter;
    T.task_clock = st->record_clock ? st->d_task_clock : nullptr;
    T.task_sm = st->record_clock ? st->d_task_sm : nullptr;
    CU(cudaMemsetAsync(st->d_counter, 0, sizeof(int), st->stream));
    int nw = st->warps < 2 ? 2 : st->warps;
    const int tc = st->tab_global ? 0 : st->ncoef, tp = st->tab_global ? 0 : st->npots;
    size_t smem = warps_smem_bytes(cap, nw, tc, tp, st->max_type, st->stages);
    while (smem > 200 * 1024 && nw > 2) {
        nw /= 2;
        smem = warps_smem_bytes(cap, nw, tc, tp, st->max_type, st->stages);
    }
    if (smem > 220 * 1024) {
        errs_register(engine_err_maxparts, "Cell too large for the sweep kernel's shared memory.", __LINE__,
                      __func__, __FILE__);
        return engine_err = engine_err_maxparts;
    }
    return st->layout ? launch_tuned_lay<1>(st, T, cap, smem, nw) : launch_tuned_lay<0>(st, T, cap, smem, nw);
}

// Records an event; inside a stream capture as an external record node, so that replaying
// the graph records it again (a plain record would stay internal to the graph).
int record_event(NbState* st, cudaEvent_t ev) {
    if (st->capturing)
        CU(cudaEventRecordWithFlags(ev, st->stream, cudaEventRecordExternal));
    else
        CU(cudaEventRecord(ev, st->stream));
    return 0;
}

// Where the particles of an evaluation live on the device: the per-evaluation slots of the
// host-buffer path, or the fixed per-cell blocks of resident steps.
struct DevView {
    const float4* xq;
    const int* pid;
    unsigned* keys;
    unsigned long long* force;
    const int* cstart;
    const int* ccount;
    size_t slots;            // slots of the force accumulators
    int cap4;                // largest cell (or cell capacity), rounded up to 4
    int cpc;                 // cells per sort block
    const unsigned long long* abort = nullptr;   // resident steps: the step's abort word
    const int* rebuild = nullptr;                // Verlet skin: sort only when *rebuild
    const int* cell_mdx = nullptr;               // Verlet skin: displacements in key units
};

DevView host_view(const NbState* st) {
    DevView V;
    V.xq = st->d_xq;
    V.pid = st->d_pid;
    V.keys = st->d_keys;
    V.force = st->d_force;
    V.cstart = st->d_cstart;
    V.ccount = st->d_ccount;
    V.slots = (size_t)st->h_cstart[st->ncells];
    V.cap4 = (st->maxcount + 3) & ~3;
    V.cpc = sort_cells_per_block(st->h_cstart[st->ncells], st->ncells);
    return V;
}

// The launches of one evaluation: zero the accumulators, sort, (compact the queue,) sweep.
// span: record ev0/ev1 around them (inside a captured graph as event nodes, so that they
// time the device work and not the host's launch).
int issue_kernels(NbState* st, const DevView& V, bool span = true) {
    if (span) {
        const int rc = record_event(st, st->ev0);
        if (rc < 0) return rc;
    }
    CU(cudaMemsetAsync(V.force, 0, sizeof(unsigned long long) * 3 * V.slots, st->stream));
    CU(cudaMemsetAsync(st->d_acc, 0, sizeof(unsigned long long) * kAccCount, st->stream));
    CU(cudaMemsetAsync(st->d_cell_epot, 0, sizeof(unsigned long long) * 2 * st->ncells, st->stream));
    const int cap = V.cap4;
    if (cap == 0) {                   // no particles: nothing to launch
        int rc = record_event(st, st->evs0);
        if (rc == 0) rc = record_event(st, st->evs1);
        if (rc == 0 && span) rc = record_event(st, st->ev1);
        return rc;
    }
    int rc0 = launch_sort(V.xq, V.cstart, V.ccount, st->d_cmask, V.keys, st->d_cscale, st->ncells, V.cpc, cap,
                          st->d_acc, V.abort, st->capturing, st->stream, V.rebuild);
    if (rc0 < 0) return rc0;

    Params P;
    P.xq = V.xq;
    P.pid = V.pid;
    P.keys = V.keys;
    P.cstart = V.cstart;
    P.ccount = V.ccount;
    P.force = V.force;
    P.acc = st->d_acc;
    P.cell_epot = st->d_cell_epot;
    P.cell_vir = st->d_cell_epot + st->ncells;
    P.tasks = st->d_tasks;
    P.tshift = st->d_tshift;
    P.ntasks = st->ntasks;
    P.coef = st->d_coef;
    P.potinfo = st->d_potinfo;
    P.potn = st->d_potn;
    P.potidx = st->d_potidx;
    P.max_type = st->max_type;
    P.npots = st->npots;
    P.ncoef = st->ncoef;
    P.emask = st->d_emask;
    P.exoff = st->d_exoff;
    P.exlist = st->d_exlist;
    P.cutoff2 = st->cut2p;
    P.cutoff2s = st->cut2s;
    P.unsorted = st->unsorted;
    P.abort = V.abort;
    P.qid = st->d_qid;
    P.ep_pot = st->ep_pot;
    P.tab_global = st->tab_global;
    P.tiny = tiny_tasks_of(st);
    P.cell_mdx = V.cell_mdx;

    const bool f32 = st->plain && st->fp32acc;
    if (f32) {
        if (st->force32_slots < V.slots) {           // grown on a direct launch, never in a capture
            if (st->capturing) {
                errs_register(engine_err_cuda, "FP32 force buffer too small inside a stream capture.", __LINE__,
                              __func__, __FILE__);
                return engine_err = engine_err_cuda;
            }
            if (st->d_force32) CU(cudaFree(st->d_force32));
            st->d_force32 = nullptr;
            st->force32_slots = 0;
            CU(cudaMalloc(&st->d_force32, sizeof(float) * 3 * V.slots));
            st->force32_slots = V.slots;
            st->buf_gen++;                           // graphs holding the old buffer are re-made
        }
        CU(cudaMemsetAsync(st->d_force32, 0, sizeof(float) * 3 * V.slots, st->stream));
        P.force32 = st->d_force32;
    }
    int rc = record_event(st, st->evs0);
    if (rc < 0) return rc;
    rc = st->plain ? launch_plain(st, P, cap) : launch_tuned(st, P, cap);
    if (rc < 0) return rc;
    rc = record_event(st, st->evs1);
    if (rc < 0) return rc;
    if (f32) {
        const size_t n = 3 * V.slots;
        const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)st->sm_count * 8);
        force32_to_fixed<<<blocks, 256, 0, st->stream>>>(st->d_force32, V.force, n, st->d_acc, V.abort);
        CU(cudaGetLastError());
    }
    if (!span) return 0;
    return record_event(st, st->ev1);
}

int issue_kernels(NbState* st) { return issue_kernels(st, host_view(st)); }

void drop_graph(NbState* st) {
    if (st->graph_exec) cudaGraphExecDestroy(st->graph_exec);
    if (st->graph) cudaGraphDestroy(st->graph);
    st->graph_exec = nullptr;
    st->graph = nullptr;
    st->graph_key = -1;
}

// Everything the captured launches depend on besides the device buffers' contents.
long long launch_key(const NbState* st) {
    long long k = st->h_cstart[st->ncells];                    // slots
    k = k * 1031 + st->maxcount;
    k = k * 131 + st->buf_gen;
    k = k * 17 + st->warps;
    k = k * 17 + st->window;
    k = k * 3 + st->layout;
    k = k * 3 + st->stages;
    k = k * 3 + (st->occupancy == 640 ? 0 : st->occupancy == 768 ? 1 : 2);
    k = k * 3 + st->plain;
    k = k * 3 + st->record_clock;
    k = k * 2 + st->fp32acc;
    return k;
}

// One evaluation on the device.  With graphs enabled, the first evaluation of a launch
// configuration runs directly (it sets the kernels' attributes and sizes the grid), the
// second captures the launches into a graph, and later ones replay it.
int launch_kernels(NbState* st) {
    if (!st->use_graph) return issue_kernels(st);
    const long long key = launch_key(st);
    if (st->graph_exec != nullptr && st->graph_key == key) {
        CU(cudaGraphLaunch(st->graph_exec, st->stream));
        return 0;
    }
    if (st->prepared_key != key) {
        drop_graph(st);
        st->prepared_key = key;
        return issue_kernels(st);
    }
    drop_graph(st);
    CU(cudaStreamBeginCapture(st->stream, cudaStreamCaptureModeThreadLocal));
    st->capturing = true;
    int rc = issue_kernels(st);
    st->capturing = false;
    cudaGraph_t g = nullptr;
    const cudaError_t end = cudaStreamEndCapture(st->stream, &g);
    if (rc < 0) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    CU(end);
    st->graph = g;
    CU(cudaGraphInstantiate(&st->graph_exec, g, 0));
    st->graph_key = key;
    CU(cudaGraphLaunch(st->graph_exec, st->stream));
    return 0;
}

// Reads back the accumulators: per-engine energies and virials into each engine's stats
// and cells, totals into st->bstats.
// sums: each engine's fixed-point energy and virial sums when the caller has set the
// cells' energies already (the resident download does it while rebuilding the cells), else
// nullptr.
int finish_stats(NbState* st, const std::vector<long long>* sums = nullptr) {
    const unsigned long long* a = st->h_acc;
    const unsigned long long* cvir = st->h_cell_epot + st->ncells;
    const size_t ne = st->engines.size();
    // The cells' energies and each engine's fixed-point sums (host threads over ranges of
    // engines, or of one engine's cells; integer sums, so the same in any order).
    std::vector<long long> esums(ne, 0), vsums(ne, 0);
    if (sums != nullptr) {
        for (size_t k = 0; k < ne; k++) {
            esums[k] = (*sums)[2 * k];
            vsums[k] = (*sums)[2 * k + 1];
        }
    }
    auto cell_range = [&](size_t k, int b, int e, long long& es, long long& vs) {
        struct space* s = &st->engines[k]->s;
        for (int c = b; c < e; c++) {
            const long long v = (long long)st->h_cell_epot[st->cell_off[k] + c];
            es += v;
            vs += (long long)cvir[st->cell_off[k] + c];
            s->cells[c].epot = (double)v / kEnergyScale;
        }
    };
    if (sums != nullptr) {
    } else if (ne > 1) {
        HostPool::get().run((int)ne, std::max(1, kCellPassGrain * (int)ne / std::max(1, st->ncells)),
                            [&](int, int b, int e) {
                                for (int k = b; k < e; k++)
                                    cell_range(k, 0, st->engines[k]->s.nr_cells, esums[k], vsums[k]);
                            });
    } else if (ne == 1) {
        const int parts = HostPool::get().threads();
        std::vector<long long> ep(parts, 0), vp(parts, 0);
        HostPool::get().run(st->engines[0]->s.nr_cells, kCellPassGrain,
                            [&](int part, int b, int e) { cell_range(0, b, e, ep[part], vp[part]); });
        for (int q = 0; q < parts; q++) {
            esums[0] += ep[q];
            vsums[0] += vp[q];
        }
    }
    long long etot = 0, vtot = 0;
    for (size_t k = 0; k < ne; k++) {
        struct engine* e = st->engines[k];
        struct space* s = &e->s;
        const long long esum = esums[k], vsum = vsums[k];
        etot += esum;
        vtot += vsum;
        e->stats.epot = (double)esum / kEnergyScale;
        e->stats.virial = -(double)vsum / kEnergyScale;
        e->stats.status = (int)a[kAccStatus];
        s->epot_nonbond += e->stats.epot;
        if (st->engines.size() == 1) {
            e->stats.pairs = (int64_t)a[kAccPairs];
            e->stats.excluded = (int64_t)a[kAccExcl];
            e->stats.candidates = (int64_t)a[kAccCand];
        } else {                               // counts are kept for the batch only
            e->stats.pairs = e->stats.excluded = e->stats.candidates = -1;
        }
    }
    st->bstats.epot = (double)etot / kEnergyScale;
    st->bstats.virial = -(double)vtot / kEnergyScale;
    st->bstats.pairs = (int64_t)a[kAccPairs];
    st->bstats.excluded = (int64_t)a[kAccExcl];
    st->bstats.candidates = (int64_t)a[kAccCand];
    st->bstats.status = (int)a[kAccStatus];
    if (a[kAccStatus] != 0) {
        const char* msg = (a[kAccStatus] & kStatusCellOverflow)   ? "Max. number of parts per cell exceeded."
                          : (a[kAccStatus] & kStatusCopyTimeout)  ? "Bulk copy into shared memory timed out."
                          : (a[kAccStatus] & kStatusTableIndex)   ? "Pair distance beyond the potential table."
                          : (a[kAccStatus] & kStatusNonFinite)    ? "Non-finite particle position or velocity."
                                                                   : "Fixed-point force overflow.";
        int code = (a[kAccStatus] & kStatusCellOverflow) ? engine_err_maxparts : engine_err_cuda;
        errs_register(code, msg, __LINE__, __func__, __FILE__);
        return engine_err = code;
    }
    return 0;
}

void res_free(NbState* st);
int refresh_charges(NbState* st);

void state_free(NbState* st) {
    if (st == nullptr) return;
    for (NbState* g : st->groups) state_free(g);
    st->groups.clear();
    cudaSetDevice(st->device);
    drop_graph(st);
    res_free(st);
    void* dev[] = {st->d_xq, st->d_pid, st->d_keys, st->d_force, st->d_cstart, st->d_ccount, st->d_cmask,
                   st->d_cscale, st->d_acc, st->d_cell_epot, st->d_tasks, st->d_tshift, st->d_coef, st->d_potinfo,
                   st->d_potn, st->d_potidx, st->d_emask, st->d_exoff, st->d_exlist, st->d_order,
                   st->d_counter, st->d_task_clock, st->d_task_sm, st->d_forcef, st->d_queue,
                   st->d_qcount, st->d_bsum, st->d_qid, st->d_force32, st->r_elog, st->r_eacc};
    for (void* p : dev) cudaFree(p);
    void* host[] = {st->h_xq, st->h_pid, st->h_cstart, st->h_force, st->h_cell_epot, st->h_acc};
    for (void* p : host) cudaFreeHost(p);
    if (st->ev0) cudaEventDestroy(st->ev0);
    if (st->ev1) cudaEventDestroy(st->ev1);
    if (st->evs0) cudaEventDestroy(st->evs0);
    if (st->evs1) cudaEventDestroy(st->evs1);
    for (cudaEvent_t ev : st->chunk_ev) cudaEventDestroy(ev);
    if (st->own_stream) cudaStreamDestroy(st->own_stream);
    sched_free(st->sched);
    delete st;
}

// Same table contents (the batch evaluates every engine with engine 0's tables).
bool same_table(const struct potential* p, const struct potential* q) {
    if (p == q) return true;
    if (p == nullptr || q == nullptr) return false;
    if (p->n != q->n || std::memcmp(p->alpha, q->alpha, sizeof(p->alpha)) != 0) return false;
    return std::memcmp(p->c, q->c, sizeof(float) * (size_t)(p->n + 1) * potential_chunk) == 0;
}

// Builds the device state of st->engines: tables, tasks, queue order, cell data, exclusions.
int load_state(NbState* st) {
    struct engine* e0 = st->engines[0];
    const size_t ne = st->engines.size();
    const int mt = e0->max_type;
    st->cell_off.assign(ne + 1, 0);
    st->id_off.assign(ne + 1, 0);
    for (size_t k = 0; k < ne; k++) {                 // checked before any device call
        struct engine* e = st->engines[k];
        if (e->device != e0->device || e->max_type != mt || e->s.cutoff != e0->s.cutoff ||
            (e->flags & engine_flag_unsorted) != (e0->flags & engine_flag_unsorted)) {
            errs_register(engine_err_range, "Engines of a batch differ in device, types, cutoff or flags.", __LINE__,
                          __func__, __FILE__);
            return engine_err = engine_err_range;
        }
        for (int ij = 0; ij < mt * mt; ij++)
            if (!same_table(e->p[ij], e0->p[ij])) {
                errs_register(engine_err_potential, "Engines of a batch differ in their potentials.", __LINE__,
                              __func__, __FILE__);
                return engine_err = engine_err_potential;
            }
        if (!same_table(e->ep, e0->ep)) {
            errs_register(engine_err_potential, "Engines of a batch differ in their explicit electrostatics.",
                          __LINE__, __func__, __FILE__);
            return engine_err = engine_err_potential;
        }
        st->cell_off[k + 1] = st->cell_off[k] + e->s.nr_cells;
        st->id_off[k + 1] = st->id_off[k] + (e->s.size_parts > 0 ? e->s.size_parts : 1);
    }
    st->ncells = st->cell_off[ne];
    st->flat_cells.clear();
    for (struct engine* e : st->engines)
        for (int c = 0; c < e->s.nr_cells; c++) st->flat_cells.push_back(&e->s.cells[c]);
    st->device = e0->device;
    CU(cudaSetDevice(st->device));
    CU(cudaStreamCreateWithFlags(&st->own_stream, cudaStreamNonBlocking));
    st->stream = st->own_stream;
    CU(cudaEventCreate(&st->ev0));
    CU(cudaEventCreate(&st->ev1));
    CU(cudaEventCreate(&st->evs0));
    CU(cudaEventCreate(&st->evs1));
    CU(cudaDeviceGetAttribute(&st->sm_count, cudaDevAttrMultiProcessorCount, st->device));
    nb_sweep_scales(&e0->s, &st->bias, &st->dscale, &st->dmaxdist);
    const float cutf = (float)e0->s.cutoff;
    st->cut2p = cutf * cutf;
    st->cut2s = (float)e0->s.cutoff2;
    st->unsorted = (e0->flags & engine_flag_unsorted) ? 1 : 0;

    float axes[13][3];
    for (int sid = 0; sid < 13; sid++) sort_axis(sid, axes[sid]);
    CU(cudaMemcpyToSymbol(c_axes, axes, sizeof(axes)));

    // Potential tables: one copy of every distinct table, type pair -> table index.
    std::vector<struct potential*> uniq;
    std::vector<int> potidx((size_t)mt * mt, -1);
    for (int i = 0; i < mt; i++)
        for (int j = 0; j < mt; j++) {
            struct potential* p = e0->p[i * mt + j];
            if (p == nullptr) continue;
            int k = 0;
            while (k < (int)uniq.size() && uniq[k] != p) k++;
            if (k == (int)uniq.size()) uniq.push_back(p);
            potidx[i * mt + j] = k;
        }
    // The explicit electrostatic potential, if any, is one more table.
    st->ep_pot = -1;
    if (e0->ep != nullptr) {
        int k = 0;
        while (k < (int)uniq.size() && uniq[k] != e0->ep) k++;
        if (k == (int)uniq.size()) uniq.push_back(e0->ep);
        st->ep_pot = k;
    }
    std::vector<float> coef;
    std::vector<float4> potinfo;
    std::vector<int> potn;
    for (struct potential* p : uniq) {
        int off = (int)coef.size();
        coef.insert(coef.end(), p->c, p->c + (size_t)(p->n + 1) * potential_chunk);
        // w: offset of the table's chunk 0 (low 20 bits) and its last chunk index n (high 12)
        potinfo.push_back(make_float4(p->alpha[0], p->alpha[1], p->alpha[2], bits_as_float(off | (p->n << 20))));
        potn.push_back(p->n);
    }
    if (coef.size() >= (1u << 20)) {
        errs_register(engine_err_potential, "Potential tables exceed 2^20 floats.", __LINE__, __func__, __FILE__);
        return engine_err = engine_err_potential;
    }
    st->npots = (int)uniq.size();
    st->one_pot = (uniq.size() == 1) && std::all_of(potidx.begin(), potidx.end(), [](int v) { return v == 0; }) &&
                  st->ep_pot < 0;
    // Tables of more than 24 KB (many type pairs) would crowd the sweep's shared memory; they
    // are read from global memory instead, as they are with explicit electrostatics.
    st->tab_global = (st->ep_pot >= 0 || coef.size() * sizeof(float) > 24 * 1024) ? 1 : 0;
    st->ncoef = (int)coef.size();
    st->max_type = mt;
    if (coef.empty()) coef.push_back(0.f);
    if (potinfo.empty()) { potinfo.push_back(make_float4(0, 0, 0, 0)); potn.push_back(0); }
    if (dev_alloc(&st->d_coef, coef.size()) || dev_alloc(&st->d_potinfo, potinfo.size()) ||
        dev_alloc(&st->d_potn, potn.size()) || dev_alloc(&st->d_potidx, potidx.size()))
        return engine_err_cuda;
    CU(cudaMemcpy(st->d_coef, coef.data(), coef.size() * sizeof(float), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(st->d_potinfo, potinfo.data(), potinfo.size() * sizeof(float4), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(st->d_potn, potn.data(), potn.size() * sizeof(int), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(st->d_potidx, potidx.data(), potidx.size() * sizeof(int), cudaMemcpyHostToDevice));

    // Task list with the reference's per-pair shift, discretised shift norm and sweep
    // bound; cells: sort-direction masks and sort scales.
    int ntasks = 0;
    for (struct engine* e : st->engines) ntasks += e->s.nr_tasks;
    st->ntasks = ntasks;
    std::vector<TaskRec> tasks(ntasks > 0 ? ntasks : 1, TaskRec{0, 0, -1, 0});
    std::vector<float4> tshift(tasks.size(), make_float4(0, 0, 0, 0));
    std::vector<unsigned> cmask(st->ncells > 0 ? st->ncells : 1, 0u);
    std::vector<float2> cscale(cmask.size(), make_float2(0.f, 0.f));
    std::vector<double> cost(tasks.size(), 0.0);
    int empty = 0;
    for (size_t k = 0, t0 = 0; k < ne; k++) {
        struct space* s = &st->engines[k]->s;
        const int c0 = st->cell_off[k];
        float bias, dscale;
        int dmax;
        nb_sweep_scales(s, &bias, &dscale, &dmax);
        for (int c = 0; c < s->nr_cells; c++) {
            cmask[c0 + c] = s->cells[c].sortmask;
            cscale[c0 + c] = make_float2(dscale, bias);
            empty += s->cells[c].count == 0;
        }
        for (int t = 0; t < s->nr_tasks; t++) {
            const struct task* tk = &s->tasks[t];
            TaskRec r;
            if (tk->type == task_type_self) {
                r = TaskRec{c0 + tk->i, c0 + tk->i, -1, dmax << 16};
            } else {
                float sh[3];
                int dn, ci, cj;
                const int sid = nb_task_shift(s, t, dscale, sh, &dn, &ci, &cj);
                r = TaskRec{c0 + ci, c0 + cj, sid, dn | (dmax << 16)};
                tshift[t0 + t] = make_float4(sh[0], sh[1], sh[2], 0.f);
            }
            tasks[t0 + t] = r;
            // Initial queue order by decreasing estimated cost, the reference's cell-pair
            // weight (src/engine.c:574-576, 643-699): count_i*count_j times 0.50004 (face),
            // 0.16176 (edge) or 0.036213 (corner) neighbours, n^2 - n for a cell with itself.
            cost[t0 + t] = task_weight(r.sid, s->cells[r.ci - c0].count, s->cells[r.cj - c0].count);
        }
        t0 += s->nr_tasks;
    }
    if (dev_alloc(&st->d_tasks, tasks.size()) || dev_alloc(&st->d_tshift, tshift.size())) return engine_err_cuda;
    CU(cudaMemcpy(st->d_tasks, tasks.data(), tasks.size() * sizeof(TaskRec), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(st->d_tshift, tshift.data(), tshift.size() * sizeof(float4), cudaMemcpyHostToDevice));
    {
        std::vector<int> order(tasks.size(), 0);
        for (int t = 0; t < ntasks; t++) order[t] = t;
        std::stable_sort(order.begin(), order.begin() + ntasks, [&](int a, int b) { return cost[a] > cost[b]; });
        st->heur_order.assign(order.begin(), order.begin() + ntasks);
        // Many small tasks per worker warp (replica batches, large systems of small cells):
        // the same costs in locality tiles, so that neighbouring cells are swept close
        // together in time and read from L2 (1-2 % faster on such systems).  With few large
        // tasks (tiles of fewer than 4) plain longest-first.
        // (sized for the most worker warps a launch shape has, 1024 threads per SM: the shape
        // is chosen later, and the small-task systems this serves run best there)
        const int tile = auto_tile(ntasks, st->sm_count, 1024);
        if (tile >= 4) {
            const std::vector<int> tiled = tiled_order(cost, ntasks, tile);
            std::copy(tiled.begin(), tiled.end(), order.begin());
        }
        const int nb = (ntasks + kQueueBlock - 1) / kQueueBlock + 1;
        if (dev_alloc(&st->d_queue, order.size()) || dev_alloc(&st->d_qcount, 1) || dev_alloc(&st->d_bsum, nb))
            return engine_err_cuda;
        st->compact = empty > 0;
        if (dev_alloc(&st->d_order, order.size()) || dev_alloc(&st->d_counter, 1) ||
            dev_alloc(&st->d_task_clock, 2 * order.size()) || dev_alloc(&st->d_task_sm, order.size()))
            return engine_err_cuda;
        CU(cudaMemcpy(st->d_order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    if (dev_alloc(&st->d_cmask, cmask.size()) || dev_alloc(&st->d_cscale, cscale.size()) ||
        dev_alloc(&st->d_cstart, st->ncells + 1) || dev_alloc(&st->d_ccount, cmask.size()) ||
        dev_alloc(&st->d_cell_epot, 2 * cmask.size()) || dev_alloc(&st->d_acc, kAccCount))
        return engine_err_cuda;
    CU(cudaMemcpy(st->d_cmask, cmask.data(), cmask.size() * sizeof(unsigned), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(st->d_cscale, cscale.data(), cscale.size() * sizeof(float2), cudaMemcpyHostToDevice));
    CU(cudaMallocHost(&st->h_cstart, sizeof(int) * (2 * st->ncells + 2)));
    CU(cudaMallocHost(&st->h_cell_epot, sizeof(unsigned long long) * (2 * st->ncells + 2)));
    CU(cudaMallocHost(&st->h_acc, sizeof(unsigned long long) * kAccCount));
    std::memset(st->h_cstart, 0, sizeof(int) * (2 * st->ncells + 2));

    // Exclusions by global particle id: a bit mask for partners at id offsets -16..16, a
    // CSR list for the rest.  Each exclusion is recorded on both particles.
    const int nid = st->id_off[ne];
    st->nid = nid;
    std::vector<std::pair<int, int>> ex;          // global ids, in range, distinct
    for (size_t k = 0; k < ne; k++) {
        struct engine* e = st->engines[k];
        const int lo = st->id_off[k], n = st->id_off[k + 1] - lo;
        for (int x = 0; x < e->nr_exclusions; x++) {
            const int a = e->exclusions[x].i, b = e->exclusions[x].j;
            if (a < 0 || b < 0 || a >= n || b >= n || a == b) continue;
            ex.emplace_back(lo + a, lo + b);
        }
    }
    st->has_excl = !ex.empty();
    st->need_pid = st->has_excl || st->ep_pot >= 0;
    if (dev_alloc(&st->d_qid, nid + 1)) return engine_err_cuda;
    refresh_charges(st);
    std::vector<unsigned> emask(nid, 0u);
    std::vector<int> cnt(nid + 1, 0);
    for (const auto& ab : ex) {
        const int a = ab.first, b = ab.second, d = b - a;
        if (d >= -16 && d <= 16) {
            emask[a] |= 1u << ((d < 0) ? d + 16 : d + 15);
            emask[b] |= 1u << ((-d < 0) ? -d + 16 : -d + 15);
        } else {
            cnt[a + 1]++;
            cnt[b + 1]++;
        }
    }
    for (int q = 0; q < nid; q++) cnt[q + 1] += cnt[q];
    std::vector<int> exlist(cnt[nid] > 0 ? cnt[nid] : 1), fill(cnt.begin(), cnt.end() - 1);
    for (const auto& ab : ex) {
        const int a = ab.first, b = ab.second, d = b - a;
        if (d >= -16 && d <= 16) continue;
        exlist[fill[a]++] = b;
        exlist[fill[b]++] = a;
    }
    if (dev_alloc(&st->d_emask, nid) || dev_alloc(&st->d_exoff, nid + 1) || dev_alloc(&st->d_exlist, exlist.size()))
        return engine_err_cuda;
    CU(cudaMemcpy(st->d_emask, emask.data(), nid * sizeof(unsigned), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(st->d_exoff, cnt.data(), (nid + 1) * sizeof(int), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(st->d_exlist, exlist.data(), exlist.size() * sizeof(int), cudaMemcpyHostToDevice));
    return 0;
}

// Charges by global particle id from the engines' host cells, to the device (explicit
// electrostatics only; other systems never read them).
int refresh_charges(NbState* st) {
    if (st->ep_pot < 0) return 0;
    st->h_qid.assign((size_t)st->nid + 1, 0.f);
    for (size_t k = 0; k < st->engines.size(); k++) {
        const struct space* sp = &st->engines[k]->s;
        for (int c = 0; c < sp->nr_cells; c++)
            for (int q = 0; q < sp->cells[c].count; q++) {
                const struct part* p = &sp->cells[c].parts[q];
                st->h_qid[(size_t)st->id_off[k] + p->id] = p->q;
            }
    }
    CU(cudaMemcpyAsync(st->d_qid, st->h_qid.data(), sizeof(float) * st->h_qid.size(), cudaMemcpyHostToDevice,
                       st->stream));
    CU(cudaStreamSynchronize(st->stream));
    return 0;
}

// Copies of the timing fields of the last evaluation into every engine's stats.
void share_times(NbState* st) {
    for (struct engine* e : st->engines) {
        e->stats.ms_kernels = st->bstats.ms_kernels;
        e->stats.ms_pack = st->bstats.ms_pack;
        e->stats.ms_device = st->bstats.ms_device;
        e->stats.ms_unpack = st->bstats.ms_unpack;
    }
}

// Packs and uploads the particles: slot layout, then chunk by chunk (pack on host threads,
// one asynchronous copy per array), so that the copy of a chunk overlaps the packing of the
// next.
int st_load_parts(NbState* st) {
    CU(cudaSetDevice(st->device));
    const double t0 = now_ms();
    if (st->ep_pot >= 0) {               // charges may have been changed on the host
        const int rc = refresh_charges(st);
        if (rc < 0) return rc;
    }
    const int slots = prepare_slots(st);
    if (slots < 0) return slots;
    const std::vector<int> bounds = chunk_bounds(st, slots);
    for (size_t q = 0; q + 1 < bounds.size(); q++) {
        const int cb = bounds[q], ce = bounds[q + 1];
        if (ce <= cb) continue;
        pack_range(st, cb, ce);
        const int s0 = st->h_cstart[cb], n = st->h_cstart[ce] - s0;
        if (n <= 0) continue;
        CU(cudaMemcpyAsync(st->d_xq + s0, st->h_xq + s0, sizeof(float4) * n, cudaMemcpyHostToDevice, st->stream));
        if (st->need_pid)
            CU(cudaMemcpyAsync(st->d_pid + s0, st->h_pid + s0, sizeof(int) * n, cudaMemcpyHostToDevice, st->stream));
    }
    const double t1 = now_ms();
    st->bstats.ms_pack = (float)(t1 - t0);
    st->bstats.ms_device = 0.f;
    CU(cudaMemcpyAsync(st->d_cstart, st->h_cstart, sizeof(int) * (st->ncells + 1), cudaMemcpyHostToDevice,
                       st->stream));
    CU(cudaMemcpyAsync(st->d_ccount, st->h_cstart + st->ncells + 1, sizeof(int) * st->ncells,
                       cudaMemcpyHostToDevice, st->stream));
    st->resident_valid = true;
    share_times(st);
    return 0;
}

// Copies forces and energies of the last evaluation back into the engines' cells.
// Forces of cells [cb, ce) from the download buffer into the cells (host threads): added,
// or, when fresh, replacing the cells' forces.
void unpack_range(NbState* st, const float* hf, int cb, int ce, bool fresh) {
    HostPool::get().run(ce - cb, cell_grain(st), [&](int, int b, int e) {
        for (int c = cb + b; c < cb + e; c++) {
            struct cell* cl = st->flat_cells[c];
            const float* f = hf + 3 * (size_t)st->h_cstart[c];
            if (fresh)
                for (int q = 0; q < cl->count; q++) {
                    cl->parts[q].f[0] = f[3 * q];
                    cl->parts[q].f[1] = f[3 * q + 1];
                    cl->parts[q].f[2] = f[3 * q + 2];
                }
            else
                for (int q = 0; q < cl->count; q++) {
                    cl->parts[q].f[0] += f[3 * q];
                    cl->parts[q].f[1] += f[3 * q + 1];
                    cl->parts[q].f[2] += f[3 * q + 2];
                }
        }
        const size_t s0 = (size_t)st->h_cstart[cb + b], s1 = (size_t)st->h_cstart[cb + e];
        evict_lines(hf + 3 * s0, sizeof(float) * 3 * (s1 - s0));
    });
}

// fresh: the evaluation's forces and energies replace those of the cells (one pass over
// the particles instead of zeroing them first); otherwise they are added.
int st_unload_parts(NbState* st, bool fresh = false) {
    CU(cudaSetDevice(st->device));
    const int slots = st->h_cstart[st->ncells];
    const double t0 = now_ms();
    if (slots > 0) {
        fixed_to_float<<<(3 * slots + 255) / 256, 256, 0, st->stream>>>(st->d_force, st->d_forcef, 3 * slots);
        CU(cudaGetLastError());
    }
    float* hf = reinterpret_cast<float*>(st->h_force);
    const std::vector<int> bounds = chunk_bounds(st, slots);
    const size_t nch = bounds.size() - 1;
    if (chunk_events(st, nch) < 0) return engine_err_cuda;
    for (size_t q = 0; q < nch; q++) {
        const int s0 = st->h_cstart[bounds[q]], n = st->h_cstart[bounds[q + 1]] - s0;
        if (n > 0)
            CU(cudaMemcpyAsync(hf + 3 * (size_t)s0, st->d_forcef + 3 * (size_t)s0, sizeof(float) * 3 * (size_t)n,
                               cudaMemcpyDeviceToHost, st->stream));
        CU(cudaEventRecord(st->chunk_ev[q], st->stream));
    }
    CU(cudaMemcpyAsync(st->h_cell_epot, st->d_cell_epot, sizeof(unsigned long long) * 2 * st->ncells,
                       cudaMemcpyDeviceToHost, st->stream));
    CU(cudaMemcpyAsync(st->h_acc, st->d_acc, sizeof(unsigned long long) * kAccCount, cudaMemcpyDeviceToHost,
                       st->stream));
    // Forces chunk by chunk as they arrive (the unpacking of one overlaps the copy of the next).
    double t_unpack = 0.0;
    for (size_t q = 0; q < nch; q++) {
        CU(cudaEventSynchronize(st->chunk_ev[q]));
        const double u0 = now_ms();
        unpack_range(st, hf, bounds[q], bounds[q + 1], fresh);
        t_unpack += now_ms() - u0;
    }
    CU(cudaStreamSynchronize(st->stream));
    const double t1 = now_ms();
    float ms = 0.f;
    // The events are unset when no evaluation ran since the last load; that error is
    // cleared here so that it does not surface at the next launch check.
    if (cudaEventElapsedTime(&ms, st->ev0, st->ev1) == cudaSuccess)
        st->bstats.ms_kernels = ms;
    else
        cudaGetLastError();
    if (fresh)
        for (struct engine* e : st->engines) {
            struct space* s = &e->s;
            s->epot = s->epot_nonbond = s->epot_bond = s->epot_angle = s->epot_dihedral = s->epot_exclusion = 0.0;
        }
    const int rc = finish_stats(st);
    st->bstats.ms_device += (float)(t1 - t0 - t_unpack);
    st->bstats.ms_unpack = (float)(t_unpack + (now_ms() - t1));
    share_times(st);
    return rc;
}

// Sort + sweep on the particles already resident on the device.
int st_resident(NbState* st) {
    if (!st->resident_valid) {
        errs_register(engine_err_cuda, "No particles resident on the device.", __LINE__, __func__, __FILE__);
        return engine_err = engine_err_cuda;
    }
    CU(cudaSetDevice(st->device));
    return launch_kernels(st);
}

int st_nonbond(NbState* st, bool fresh = false) {
    int rc = st_load_parts(st);
    if (rc < 0) return rc;
    rc = st_resident(st);
    if (rc < 0) return rc;
    return st_unload_parts(st, fresh);
}

int st_setstream(NbState* st, void* stream) {
    CU(cudaSetDevice(st->device));
    CU(cudaStreamSynchronize(st->stream));
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : st->own_stream;
    if (s != st->stream) drop_graph(st);
    st->stream = s;
    return 0;
}

int st_kernel_times(NbState* st, float* total_ms, float* sweep_ms) {
    CU(cudaSetDevice(st->device));
    CU(cudaStreamSynchronize(st->stream));
    float a = 0.f, b = 0.f;
    CU(cudaEventElapsedTime(&a, st->ev0, st->ev1));
    CU(cudaEventElapsedTime(&b, st->evs0, st->evs1));
    if (total_ms) *total_ms = a;
    if (sweep_ms) *sweep_ms = b;
    return 0;
}

int st_settune(NbState* st, int warps, int plain) {
    if (warps != 0 && warps != 1 && warps != 2 && warps != 4 && warps != 8) return engine_err_range;
    st->warps = warps ? warps : 4;
    st->plain = plain ? 1 : 0;
    return 0;
}

// Times every persistent launch shape (worker warps per block x lane layout x staging
// buffers per warp x resident threads per SM) on the resident particles, `reps`
// evaluations each after one warm-up, and keeps the fastest (median device time of sort +
// sweep).  Every shape computes the same pair set and forces within FP32 rounding.
int st_autotune(NbState* st, int reps, int* warps_out, int* layout_out, int* stages_out, int* occupancy_out,
                float* ms_out) {
    if (!st->resident_valid) {
        const int rc = st_load_parts(st);
        if (rc < 0) return rc;
    }
    CU(cudaSetDevice(st->device));
    if (reps < 1) reps = 1;
    const bool graph = st->use_graph;
    st->use_graph = false;
    st->plain = 0;
    // warps, layout, stages, threads per SM (window 4: the 8-step window was never the
    // fastest shape)
    static const int shapes[][4] = {
        {2, 0, 1, 640}, {4, 0, 1, 640}, {8, 0, 1, 640}, {2, 1, 1, 640}, {4, 1, 1, 640}, {8, 1, 1, 640},
        {2, 0, 2, 640}, {4, 0, 2, 640}, {8, 0, 2, 640}, {2, 1, 2, 640}, {4, 1, 2, 640}, {8, 1, 2, 640},
        {2, 0, 1, 768}, {4, 0, 1, 768}, {8, 0, 1, 768}, {2, 1, 1, 768}, {4, 1, 1, 768}, {8, 1, 1, 768},
        {2, 0, 1, 1024}, {4, 0, 1, 1024}, {8, 0, 1, 1024}, {2, 1, 1, 1024}, {4, 1, 1, 1024}, {8, 1, 1, 1024},
        {2, 1, 2, 1024}, {4, 1, 2, 1024}, {8, 1, 2, 1024}};
    const int nshapes = sizeof(shapes) / sizeof(shapes[0]);
    int best = -1;
    float best_ms = 0.f;
    for (int k = 0; k < nshapes; k++) {
        st->warps = shapes[k][0];
        st->layout = shapes[k][1];
        st->stages = shapes[k][2];
        st->occupancy = shapes[k][3];
        st->window = 4;
        std::vector<float> t;
        for (int r = 0; r <= reps; r++) {
            int rc = st_resident(st);
            if (rc < 0) {
                st->use_graph = graph;
                return rc;
            }
            CU(cudaEventSynchronize(st->ev1));
            float ms = 0.f;
            CU(cudaEventElapsedTime(&ms, st->ev0, st->ev1));
            if (r > 0) t.push_back(ms);
        }
        std::sort(t.begin(), t.end());
        const float med = t[t.size() / 2];
        if (best < 0 || med < best_ms) {
            best = k;
            best_ms = med;
        }
    }
    st->warps = shapes[best][0];
    st->layout = shapes[best][1];
    st->stages = shapes[best][2];
    st->occupancy = shapes[best][3];
    st->window = 4;
    st->use_graph = graph;
    const int rc = st_resident(st);           // leave the chosen shape's results resident
    if (rc < 0) return rc;
    if (warps_out) *warps_out = st->warps;
    if (layout_out) *layout_out = st->layout;
    if (stages_out) *stages_out = st->stages;
    if (occupancy_out) *occupancy_out = st->occupancy;
    if (ms_out) *ms_out = best_ms;
    return 0;
}


// ---------------------------------------------------------------- device-resident steps

void res_free(NbState* st) {
    for (int q = 0; q < 2; q++) {
        if (st->rgraph_exec[q]) cudaGraphExecDestroy(st->rgraph_exec[q]);
        if (st->rgraph[q]) cudaGraphDestroy(st->rgraph[q]);
        st->rgraph_exec[q] = nullptr;
        st->rgraph[q] = nullptr;
        st->rgraph_key[q] = st->rprepared[q] = -1;
    }
    void* dev[] = {st->r_xq[0], st->r_xq[1], st->r_v[0], st->r_v[1], st->r_pid[0], st->r_pid[1], st->r_cnt[0],
                   st->r_cnt[1], st->r_done, st->r_cstart, st->r_nstay, st->r_nmove, st->r_slot_of, st->r_nbr, st->r_cell_engine,
                   st->r_cell_h, st->r_engine_dt, st->r_engine_imass, st->r_movers, st->r_keys, st->r_force,
                   st->r_status, st->r_dense, st->r_doff, st->r_up_of};
    for (void* p : dev) cudaFree(p);
    if (st->h_dense) cudaFreeHost(st->h_dense);
    if (st->h_rcount) cudaFreeHost(st->h_rcount);
    if (st->h_up) cudaFreeHost(st->h_up);
    if (st->h_words) cudaFreeHost(st->h_words);
    {
        void* bdev[] = {st->r_bonds, st->r_bcoef, st->r_bpotinfo, st->r_bpotn, st->r_bab2, st->r_eng_cell0,
                        st->r_eng_cdim, st->r_eng_h, st->r_ebond, st->r_angles, st->r_dihedrals,
                        st->r_dihedral_te, st->r_bab};
        for (void* p : bdev) cudaFree(p);
        if (st->h_ebond) cudaFreeHost(st->h_ebond);
        st->r_bonds = nullptr;
        st->r_bcoef = nullptr;
        st->r_bpotinfo = nullptr;
        st->r_bpotn = nullptr;
        st->r_bab2 = nullptr;
        st->r_eng_cell0 = nullptr;
        st->r_eng_cdim = nullptr;
        st->r_eng_h = nullptr;
        st->r_ebond = nullptr;
        st->h_ebond = nullptr;
        st->r_angles = nullptr;
        st->r_dihedrals = nullptr;
        st->r_dihedral_te = nullptr;
        st->r_bab = nullptr;
        st->nbonds = st->nangles = st->ndihedrals = 0;
    }
    if (st->r_bsum) cudaFree(st->r_bsum);
    cudaFree(st->r_vw);
    cudaFree(st->r_oldx);
    cudaFree(st->r_cell_mdx);
    st->r_vw = nullptr;
    st->r_oldx = nullptr;
    st->r_cell_mdx = nullptr;
    st->verlet = false;
    st->h_words = nullptr;
    st->r_bsum = nullptr;
    st->r_doff = st->h_rcount = nullptr;
    st->h_up = nullptr;
    st->r_xq[0] = st->r_xq[1] = nullptr;
    st->r_v[0] = st->r_v[1] = nullptr;
    st->r_pid[0] = st->r_pid[1] = nullptr;
    st->r_cnt[0] = st->r_cnt[1] = nullptr;
    st->r_done = nullptr;
    st->r_cstart = st->r_nstay = st->r_nmove = st->r_slot_of = st->r_up_of = nullptr;
    st->r_nbr = st->r_cell_engine = nullptr;
    st->r_cell_h = nullptr;
    st->r_engine_dt = nullptr;
    st->r_engine_imass = nullptr;
    st->r_movers = nullptr;
    st->r_keys = nullptr;
    st->r_force = nullptr;
    st->r_status = nullptr;
    st->r_dense = nullptr;
    st->h_dense = nullptr;
    st->res_active = false;
}

// Places the dense upload (cell order, per-cell offsets; the global id in the velocity's w)
// into the cells' blocks, records each id's upload index (up_of) and, with explicit
// electrostatics, scatters the uploaded charges by id (dq, qid; else nullptr).
__global__ void __launch_bounds__(256) place_cells(ResidentCells RC, const float4* __restrict__ dxq,
                                                   const float4* __restrict__ dv,
                                                   const int* __restrict__ doff, const int* __restrict__ count,
                                                   float4* __restrict__ xq, float4* __restrict__ v,
                                                   int* __restrict__ pid, int* __restrict__ up_of,
                                                   const float* __restrict__ dq, float* __restrict__ qid) {
    const int lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (c >= RC.ncells) return;
    const int n = min(count[c], RC.capc);
    const size_t base = (size_t)c * RC.capc;
    for (int k = lane; k < n; k += 32) {
        const int o = doff[c] + k;
        const float4 vo = dv[o];
        const int id = __float_as_int(vo.w);
        xq[base + k] = dxq[o];
        v[base + k] = make_float4(vo.x, vo.y, vo.z, 0.f);
        pid[base + k] = id;
        up_of[id] = o;
        if (qid != nullptr) qid[id] = dq[o];
    }
}

// Every particle in cell order for the host copy (cell c from offset doff[c]): positions
// with the particle's index in the last upload (through up_of, by id) in w, then the
// velocities and the last evaluation's forces as float triples.
__global__ void __launch_bounds__(256) compact_cells(ResidentCells RC, const float4* __restrict__ xq,
                                                     const float4* __restrict__ v, const int* __restrict__ pid,
                                                     const int* __restrict__ count, const int* __restrict__ doff,
                                                     const unsigned long long* __restrict__ force, size_t np,
                                                     const int* __restrict__ up_of, float4* __restrict__ dx,
                                                     float* __restrict__ dv3, float* __restrict__ df3) {
    const int lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (c >= RC.ncells) return;
    const int n = min(count[c], RC.capc);
    const size_t base = (size_t)c * RC.capc;
    for (int k = lane; k < n; k += 32) {
        const size_t s = base + k, o = (size_t)doff[c] + k;
        if (o >= np) break;            // counts of an aborted step: nothing past the buffers
        const float4 x = xq[s], vs = v[s];
        dx[o] = make_float4(x.x, x.y, x.z, __int_as_float(up_of[pid[s]]));
        dv3[3 * o] = vs.x;
        dv3[3 * o + 1] = vs.y;
        dv3[3 * o + 2] = vs.z;
#pragma unroll
        for (int a = 0; a < 3; a++)
            df3[3 * o + a] = (float)((double)(long long)force[3 * s + a] * (1.0 / (double)kForceScale));
    }
}

ResidentCells res_cells(const NbState* st) {
    ResidentCells RC;
    RC.ncells = st->ncells;
    RC.capc = st->capc;
    RC.mcap = st->mcap;
    RC.nbr = st->r_nbr;
    RC.cell_h = st->r_cell_h;
    return RC;
}

// Per-cell kernels of the resident steps: one warp per cell, two cells per block (small
// blocks spread a few hundred cells over all 148 SMs).
constexpr int kCellWarps = 2;
constexpr int kCellThreads = 32 * kCellWarps;
int res_grid(const NbState* st) { return (st->ncells + kCellWarps - 1) / kCellWarps; }

// The engines' bonds for the device: global ids, the bond table of the two particles' types
// (bonds whose types have none are dropped, as bond_eval skips them), the engine; the
// distinct bond tables; per engine its first cell, cell grid and cell edge.
bool res_bonded(const NbState* st) { return st->nbonds + st->nangles + st->ndihedrals > 0; }

long long res_bonds_key(const NbState* st) {
    long long k = 0;
    for (struct engine* e : st->engines) k += e->bonds_gen;
    return k;
}

// Bonded terms of the resident steps: bonds (potential by the two particles' types), angles
// and dihedrals (potential by index), with global ids; the tables they use, each once.
int res_build_bonds(NbState* st) {
    const int ne = (int)st->engines.size();
    st->bonds_key = res_bonds_key(st);
    std::vector<int4> bonds, angles, dihedrals;
    std::vector<int> dihedral_te;
    std::vector<struct potential*> uniq;
    auto table_of = [&](struct potential* pot) {
        int u = 0;
        while (u < (int)uniq.size() && uniq[u] != pot) u++;
        if (u == (int)uniq.size()) uniq.push_back(pot);
        return u;
    };
    for (int k = 0; k < ne; k++) {
        struct engine* e = st->engines[k];
        const int np = e->s.nr_parts;
        auto present = [&](int id) { return id >= 0 && id < np && e->s.partlist[id] != nullptr; };
        if (e->nr_bonds > 0 && e->p_bond != nullptr) {
            const int mt = e->max_type;
            for (int b = 0; b < e->nr_bonds; b++) {
                const int i = e->bonds[b].i, j = e->bonds[b].j;
                if (!present(i) || !present(j)) continue;
                const struct part *pi = e->s.partlist[i], *pj = e->s.partlist[j];
                struct potential* pot = e->p_bond[pj->type * mt + pi->type];
                if (pot == nullptr) continue;
                bonds.push_back(make_int4(st->id_off[k] + i, st->id_off[k] + j, table_of(pot), k));
            }
        }
        for (int a = 0; a < e->nr_angles; a++) {
            const struct angle* an = &e->angles[a];
            if (!present(an->i) || !present(an->j) || !present(an->k)) continue;
            if (an->pid < 0 || an->pid >= e->nr_anglepots || e->p_angle[an->pid] == nullptr) continue;
            angles.push_back(make_int4(st->id_off[k] + an->i, st->id_off[k] + an->j, st->id_off[k] + an->k,
                                       (k << 16) | table_of(e->p_angle[an->pid])));
        }
        for (int d = 0; d < e->nr_dihedrals; d++) {
            const struct dihedral* dh = &e->dihedrals[d];
            if (!present(dh->i) || !present(dh->j) || !present(dh->k) || !present(dh->l)) continue;
            if (dh->pid < 0 || dh->pid >= e->nr_dihedralpots || e->p_dihedral[dh->pid] == nullptr) continue;
            dihedrals.push_back(
                make_int4(st->id_off[k] + dh->i, st->id_off[k] + dh->j, st->id_off[k] + dh->k, st->id_off[k] + dh->l));
            dihedral_te.push_back((k << 16) | table_of(e->p_dihedral[dh->pid]));
        }
    }
    st->nbonds = (int)bonds.size();
    st->nangles = (int)angles.size();
    st->ndihedrals = (int)dihedrals.size();
    if (st->nbonds + st->nangles + st->ndihedrals == 0) return 0;
    if ((!angles.empty() || !dihedrals.empty()) && (ne > 32767 || uniq.size() > 65535)) {
        st->nbonds = st->nangles = st->ndihedrals = 0;
        errs_register(engine_err_range, "Too many engines or bonded tables for the angle/dihedral records.",
                      __LINE__, __func__, __FILE__);
        return engine_err = engine_err_range;
    }
    std::vector<float> coef;
    std::vector<float4> info;
    std::vector<int> potn;
    std::vector<double2> ab2, ab;
    for (struct potential* p : uniq) {
        const int off = (int)coef.size();
        coef.insert(coef.end(), p->c, p->c + (size_t)(p->n + 1) * potential_chunk);
        info.push_back(make_float4(p->alpha[0], p->alpha[1], p->alpha[2], bits_as_float(off | (p->n << 20))));
        potn.push_back(p->n);
        ab2.push_back(make_double2(p->a * p->a, p->b * p->b));
        ab.push_back(make_double2(p->a, p->b));
    }
    std::vector<int> cell0(ne);
    std::vector<int4> cdim(ne);
    std::vector<double4> h(ne);
    for (int k = 0; k < ne; k++) {
        const struct space* sp = &st->engines[k]->s;
        cell0[k] = st->cell_off[k];
        cdim[k] = make_int4(sp->cdim[0], sp->cdim[1], sp->cdim[2], 0);
        h[k] = make_double4(sp->h[0], sp->h[1], sp->h[2], 0.0);
    }
    auto up = [&](auto** dst, const auto& v) -> int {
        using T = typename std::decay<decltype(v)>::type::value_type;
        CU(cudaMalloc(dst, sizeof(T) * std::max<size_t>(1, v.size())));
        if (!v.empty()) CU(cudaMemcpy(*dst, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
        return 0;
    };
    if (up(&st->r_bonds, bonds) < 0 || up(&st->r_angles, angles) < 0 || up(&st->r_dihedrals, dihedrals) < 0 ||
        up(&st->r_dihedral_te, dihedral_te) < 0 || up(&st->r_bcoef, coef) < 0 || up(&st->r_bpotinfo, info) < 0 ||
        up(&st->r_bpotn, potn) < 0 || up(&st->r_bab2, ab2) < 0 || up(&st->r_bab, ab) < 0 ||
        up(&st->r_eng_cell0, cell0) < 0 || up(&st->r_eng_cdim, cdim) < 0 || up(&st->r_eng_h, h) < 0)
        return engine_err_cuda;
    CU(cudaMalloc(&st->r_ebond, sizeof(unsigned long long) * 3 * ne));
    CU(cudaMallocHost(&st->h_ebond, sizeof(unsigned long long) * 3 * ne));
    CU(cudaMemset(st->r_ebond, 0, sizeof(unsigned long long) * 3 * ne));
    return 0;
}

// Largest cell of the engines' host cells and the particle count (host threads over
// ranges of cells).
int res_host_counts(const NbState* st, long long* n) {
    const int parts = HostPool::get().threads();
    std::vector<long long> tot(parts, 0);
    std::vector<int> mx(parts, 0);
    HostPool::get().run(st->ncells, kCellPassGrain, [&](int part, int b, int e) {
        long long t = 0;
        int m = 0;
        for (int c = b; c < e; c++) {
            const int k = st->flat_cells[c]->count;
            t += k;
            m = std::max(m, k);
        }
        tot[part] = t;
        mx[part] = m;
    });
    long long t = 0;
    int m = 0;
    for (int k = 0; k < parts; k++) {
        t += tot[k];
        m = std::max(m, mx[k]);
    }
    *n = t;
    return m;
}

// Device blocks of capc slots per cell for n particles, with the static cell data
// (block offsets, periodic neighbours, edges, engine of each cell, dt and 1/m).
int res_alloc(NbState* st, int capc, int mcap, long long n) {
    const int nc = st->ncells, ne = (int)st->engines.size(), mt = st->max_type, nid = st->nid;
    st->capc = capc;
    st->mcap = mcap;
    st->res_nparts = n;
    const size_t slots = (size_t)nc * st->capc;
    for (int q = 0; q < 2; q++) {
        CU(cudaMalloc(&st->r_xq[q], sizeof(float4) * slots));
        CU(cudaMalloc(&st->r_v[q], sizeof(float4) * slots));
        CU(cudaMalloc(&st->r_pid[q], sizeof(int) * slots));
        // Slots past a cell's count hold zeros or an earlier occupant (finite, ids in range).
        CU(cudaMemset(st->r_xq[q], 0, sizeof(float4) * slots));
        CU(cudaMemset(st->r_v[q], 0, sizeof(float4) * slots));
        CU(cudaMemset(st->r_pid[q], 0, sizeof(int) * slots));
    }
    CU(cudaMalloc(&st->r_keys, sizeof(unsigned) * 13 * slots));
    CU(cudaMalloc(&st->r_force, sizeof(unsigned long long) * 3 * slots));
    CU(cudaMemset(st->r_force, 0, sizeof(unsigned long long) * 3 * slots));
    CU(cudaMalloc(&st->r_cnt[0], sizeof(int) * (nc + 1)));
    CU(cudaMalloc(&st->r_cnt[1], sizeof(int) * (nc + 1)));
    CU(cudaMemset(st->r_cnt[1], 0, sizeof(int) * (nc + 1)));
    CU(cudaMalloc(&st->r_done, 2 * sizeof(unsigned long long)));
    CU(cudaMalloc(&st->r_cstart, sizeof(int) * (nc + 1)));
    CU(cudaMalloc(&st->r_nstay, sizeof(int) * (nc + 1)));
    CU(cudaMalloc(&st->r_nmove, sizeof(int) * (nc + 1)));
    CU(cudaMalloc(&st->r_movers, sizeof(Mover) * (size_t)nc * st->mcap));
    CU(cudaMalloc(&st->r_slot_of, sizeof(int) * (nid + 1)));
    CU(cudaMalloc(&st->r_up_of, sizeof(int) * (nid + 1)));
    CU(cudaMemset(st->r_up_of, 0xff, sizeof(int) * (nid + 1)));     // -1: not uploaded
    CU(cudaMalloc(&st->r_nbr, sizeof(int) * 27 * (size_t)nc));
    CU(cudaMalloc(&st->r_cell_h, sizeof(float4) * (nc + 1)));
    CU(cudaMalloc(&st->r_cell_engine, sizeof(int) * (nc + 1)));
    CU(cudaMalloc(&st->r_engine_dt, sizeof(float) * ne));
    CU(cudaMalloc(&st->r_engine_imass, sizeof(double) * (size_t)ne * mt));
    CU(cudaMalloc(&st->r_status, sizeof(unsigned long long)));
    CU(cudaMalloc(&st->r_dense, sizeof(float4) * 3 * (size_t)(n + 1)));
    CU(cudaMallocHost(&st->h_dense, sizeof(float4) * 3 * (size_t)(n + 1)));
    CU(cudaMallocHost(&st->h_up, sizeof(float4) * 2 * (size_t)(n + 1)));
    CU(cudaMalloc(&st->r_doff, sizeof(int) * (nc + 1)));
    CU(cudaMallocHost(&st->h_rcount, sizeof(int) * (2 * nc + 2)));
    CU(cudaMalloc(&st->r_bsum, sizeof(int) * ((nc + kScanBlock - 1) / kScanBlock + 1)));
    CU(cudaMallocHost(&st->h_words, 4 * sizeof(unsigned long long)));
    st->verlet = true;
    for (struct engine* e : st->engines) st->verlet = st->verlet && (e->flags & engine_flag_verlet);
    if (st->verlet) {
        // skin = min h - cutoff (src/engine.c:211), the smallest over the engines
        float skin = INFINITY;
        for (struct engine* e : st->engines)
            skin = std::min(skin, (float)(std::min(e->s.h[0], std::min(e->s.h[1], e->s.h[2])) - e->s.cutoff));
        st->verlet_skin = skin;
        CU(cudaMalloc(&st->r_vw, 4 * sizeof(int)));
        CU(cudaMemset(st->r_vw, 0, 4 * sizeof(int)));
        CU(cudaMalloc(&st->r_oldx, sizeof(float4) * slots));
        CU(cudaMemset(st->r_oldx, 0, sizeof(float4) * slots));
        CU(cudaMalloc(&st->r_cell_mdx, sizeof(int) * (nc + 1)));
        CU(cudaMemset(st->r_cell_mdx, 0, sizeof(int) * (nc + 1)));
    }

    std::vector<int> cstart(nc + 1), nbr(27 * (size_t)nc), cell_engine(nc);
    std::vector<float4> cell_h(nc);
    std::vector<float> edt(ne);
    std::vector<double> imass((size_t)ne * mt, 0.0);
    for (int c = 0; c <= nc; c++) cstart[c] = (int)((size_t)c * st->capc);
    for (int k = 0; k < ne; k++) {
        struct engine* e = st->engines[k];
        struct space* sp = &e->s;
        edt[k] = (float)e->dt;
        for (int t = 0; t < mt && t < e->max_type; t++) imass[(size_t)k * mt + t] = e->types[t].imass;
        for (int c = 0; c < sp->nr_cells; c++) {
            const int g = st->cell_off[k] + c;
            const int* loc = sp->cells[c].loc;
            cell_engine[g] = k;
            cell_h[g] = make_float4((float)sp->h[0], (float)sp->h[1], (float)sp->h[2], 0.f);
            for (int d = 0; d < 27; d++) {
                const int dl[3] = {d / 9 - 1, (d / 3) % 3 - 1, d % 3 - 1};
                int nl[3];
                for (int j = 0; j < 3; j++) nl[j] = (loc[j] + dl[j] + sp->cdim[j]) % sp->cdim[j];
                nbr[(size_t)g * 27 + d] = st->cell_off[k] + space_cellid(sp, nl[0], nl[1], nl[2]);
            }
        }
    }
    CU(cudaMemcpy(st->r_cstart, cstart.data(), sizeof(int) * (nc + 1), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(st->r_nbr, nbr.data(), sizeof(int) * nbr.size(), cudaMemcpyHostToDevice));
    CU(cudaMemcpy(st->r_cell_engine, cell_engine.data(), sizeof(int) * nc, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(st->r_cell_h, cell_h.data(), sizeof(float4) * nc, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(st->r_engine_dt, edt.data(), sizeof(float) * ne, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(st->r_engine_imass, imass.data(), sizeof(double) * imass.size(), cudaMemcpyHostToDevice));
    st->up_aux.assign((size_t)n + 1, NbState::UpAux{0, 0.f, 0, 0, 0});
    st->res_active = true;
    return res_build_bonds(st);
}

// Pipeline chunks of an engine_step transfer of np particles, 1 to st->max_chunks (8; fewer
// for the groups of a grouped batch step, whose groups already overlap one another).
int res_chunks(const NbState* st, size_t np) {
    return (int)std::max(1LL, std::min((long long)st->max_chunks, (long long)np / copy_chunk_parts()));
}

// The engines' host cells into side 0 of the device blocks (the caller has checked that
// every cell fits): positions, velocities and ids packed in cell order by the host threads,
// one copy each, then placed into the blocks on the device.
int res_upload(NbState* st) {
    const int nc = st->ncells, ne = (int)st->engines.size();
    int* cnt = st->h_rcount;
    int* off = st->h_rcount + nc + 1;
    HostPool::get().run(nc, kCellPassGrain, [&](int, int b, int e) {
        for (int c = b; c < e; c++) cnt[c] = st->flat_cells[c]->count;
    });
    off[0] = 0;
    for (int c = 0; c < nc; c++) off[c + 1] = off[c] + cnt[c];
    const size_t np = (size_t)st->res_nparts;
    float4* hx = st->h_up;
    float4* hv = st->h_up + np;
    // charges for explicit electrostatics: through the download buffers past the 10 np
    // floats a download uses (scattered by id on the device, in place_cells)
    float* hq = st->ep_pot >= 0 ? reinterpret_cast<float*>(st->h_dense) + 10 * np : nullptr;
    float* dq = reinterpret_cast<float*>(st->r_dense) + 10 * np;
    const double t0 = now_ms();
    // Chunks of cells with about equal particle counts: each chunk's copies overlap the
    // packing of the next.
    const int K = res_chunks(st, np);
    std::vector<int> bounds(K + 1, nc);
    bounds[0] = 0;
    for (int k = 1; k < K; k++)
        bounds[k] = (int)(std::lower_bound(off, off + nc + 1, (int)(np * k / K)) - off);
    for (int k = 0; k < K; k++) {
    const int c0 = bounds[k], c1 = bounds[k + 1];
    HostPool::get().run(c1 - c0, cell_grain(st), [&](int, int rb, int re) {
        const int cb = c0 + rb, ce = c0 + re;
        for (int c = cb; c < ce; c++) {
            // many small cells (each its own parts array): fetch the cell records and the
            // particles a few cells ahead
            if (c + 8 < ce) __builtin_prefetch(st->flat_cells[c + 8]);
            if (c + 4 < ce) __builtin_prefetch(st->flat_cells[c + 4]->parts);
            const struct cell* cl = st->flat_cells[c];
            const size_t k = std::upper_bound(st->cell_off.begin(), st->cell_off.end(), c) - st->cell_off.begin() - 1;
            for (int q = 0; q < cl->count; q++) {
                const struct part* p = &cl->parts[q];
                const int gid = st->id_off[k] + p->id;
                const size_t o = (size_t)off[c] + q;
                store_nt(hx + o, make_float4(p->x[0], p->x[1], p->x[2], bits_as_float((int)p->type)));
                store_nt(hv + o, make_float4(p->v[0], p->v[1], p->v[2], bits_as_float(gid)));
                st->up_aux[o] = NbState::UpAux{gid, p->q, p->vid, p->type, p->flags};
                if (hq != nullptr) store_nt(hq + o, p->q);
            }
        }
        fence_nt();
    });
    const size_t q0 = (size_t)off[c0], q1 = (size_t)off[c1];
    if (q1 > q0) {
        CU(cudaMemcpyAsync(st->r_dense + q0, hx + q0, sizeof(float4) * (q1 - q0), cudaMemcpyHostToDevice,
                           st->stream));
        CU(cudaMemcpyAsync(st->r_dense + np + q0, hv + q0, sizeof(float4) * (q1 - q0), cudaMemcpyHostToDevice,
                           st->stream));
        if (hq != nullptr)
            CU(cudaMemcpyAsync(dq + q0, hq + q0, sizeof(float) * (q1 - q0), cudaMemcpyHostToDevice, st->stream));
    }
    }
    st->bstats.ms_pack = (float)(now_ms() - t0);
    st->res_engine_n.assign(ne, 0);
    for (int k = 0; k < ne; k++) st->res_engine_n[k] = off[st->cell_off[k + 1]] - off[st->cell_off[k]];
    CU(cudaMemcpyAsync(st->r_cnt[0], cnt, sizeof(int) * nc, cudaMemcpyHostToDevice, st->stream));
    CU(cudaMemcpyAsync(st->r_doff, off, sizeof(int) * (nc + 1), cudaMemcpyHostToDevice, st->stream));
    CU(cudaMemsetAsync(st->r_status, 0, sizeof(unsigned long long), st->stream));
    CU(cudaMemsetAsync(st->r_done, 0, 2 * sizeof(unsigned long long), st->stream));
    if (st->verlet) {                  // fresh positions: the first step re-bins and sorts
        static const int first[2] = {1, 0};
        CU(cudaMemcpyAsync(st->r_vw, first, sizeof(first), cudaMemcpyHostToDevice, st->stream));
    }
    const ResidentCells RC = res_cells(st);
    place_cells<<<res_grid(st), kCellThreads, 0, st->stream>>>(RC, st->r_dense, st->r_dense + np,
                                                               st->r_doff, st->r_cnt[0], st->r_xq[0], st->r_v[0],
                                                               st->r_pid[0], st->r_up_of, dq,
                                                               hq != nullptr ? st->d_qid : nullptr);
    CU(cudaGetLastError());
    slot_of_ids<<<res_grid(st), kCellThreads, 0, st->stream>>>(RC, st->r_pid[0], st->r_cnt[0], st->r_slot_of, nullptr);
    CU(cudaGetLastError());
    st->res_done = st->res_pairs = 0;
    st->rside = 0;
    st->res_dirty = false;
    return 0;
}

// Uploads the engines' particles into the device cells.  margin: spare slots per cell
// beyond the largest (negative: 8; the sweep's shared-memory slices are sized by the block,
// so a small margin keeps its occupancy, and an overflow re-blocks with twice the margin);
// mcap: leavers per cell and step.
int st_resident_begin(NbState* st, int margin, int mcap) {
    CU(cudaSetDevice(st->device));
    CU(cudaStreamSynchronize(st->stream));
    long long n = 0;
    const int maxc = res_host_counts(st, &n);
    if (maxc > kMaxPartsPerCell) {
        errs_register(engine_err_maxparts, "Max. number of parts per cell exceeded.", __LINE__, __func__, __FILE__);
        return engine_err = engine_err_maxparts;
    }
    if (margin < 0) margin = 8;
    margin = std::max(margin, 4);
    const int capc = std::min(kMaxPartsPerCell, (maxc + margin + 3) & ~3);
    res_free(st);
    int rc = res_alloc(st, capc, std::max(mcap, 16), n);
    if (rc < 0) return rc;
    st->res_margin = margin;
    rc = res_upload(st);
    if (rc < 0) return rc;
    CU(cudaStreamSynchronize(st->stream));
    st->res_done_total = st->res_pairs_total = 0;
    st->res_regrows = 0;
    return 0;
}

// A fresh start of resident steps: the energy log's step numbers restart from 1.
int elog_restart(NbState* st) {
    if (st->elog_cap <= 0) return 0;
    const unsigned long long zero = 0ull;
    CU(cudaMemset(st->r_elog, 0, sizeof(unsigned long long) * 4 * (size_t)st->elog_cap));
    CU(cudaMemcpy(st->r_eacc + 1, &zero, sizeof(zero), cudaMemcpyHostToDevice));
    return 0;
}

// The launches of one resident step: re-binning into the other side, the force evaluation,
// the integration, the rigid constraints.
int res_issue_step(NbState* st) {
    const int r = st->rside, o = 1 - r;
    int rc = record_event(st, st->ev0);
    if (rc < 0) return rc;
    const ResidentCells RC = res_cells(st);
    const int grid = res_grid(st);
    rebin_split<<<grid, kCellThreads, 0, st->stream>>>(RC, st->r_xq[r], st->r_v[r], st->r_pid[r], st->r_cnt[r], st->r_xq[o],
                                              st->r_v[o], st->r_pid[o], st->r_nstay, st->r_nmove, st->r_movers,
                                              st->r_status, st->verlet ? st->r_vw : nullptr);
    bool rigid = false;
    for (struct engine* e : st->engines) rigid = rigid || e->nr_rigids > 0;
    rebin_gather<<<grid, kCellThreads, 0, st->stream>>>(RC, st->r_movers, st->r_nstay, st->r_nmove, st->r_xq[o], st->r_v[o],
                                               st->r_pid[o], st->r_cnt[o], st->r_status,
                                               (rigid || res_bonded(st)) ? st->r_slot_of : nullptr);
    CU(cudaGetLastError());
    const unsigned vblocks = (unsigned)(((size_t)st->ncells * st->capc + 255) / 256);
    if (st->verlet) {
        verlet_mark<<<vblocks, 256, 0, st->stream>>>(RC, st->r_cnt[o], st->r_xq[o], st->r_oldx, st->r_cell_mdx,
                                                     st->r_vw, st->r_status);
        CU(cudaGetLastError());
    }
    DevView V;
    V.rebuild = st->verlet ? st->r_vw : nullptr;
    V.cell_mdx = st->verlet ? st->r_cell_mdx : nullptr;
    V.xq = st->r_xq[o];
    V.pid = st->r_pid[o];
    V.keys = st->r_keys;
    V.force = st->r_force;
    V.cstart = st->r_cstart;
    V.ccount = st->r_cnt[o];
    V.abort = st->r_status;
    V.slots = (size_t)st->ncells * st->capc;
    V.cap4 = st->capc;
    V.cpc = st->res_nparts <= 32LL * st->ncells ? kSortWarps : 1;   // one warp per small cell
    rc = issue_kernels(st, V, false);
    if (rc < 0) return rc;
    if (res_bonded(st)) {              // the bonded forces join the sweep's before the update
        CU(cudaMemsetAsync(st->r_ebond, 0, sizeof(unsigned long long) * 3 * st->engines.size(), st->stream));
        BondArgs B;
        B.bonds = st->r_bonds;
        B.nbonds = st->nbonds;
        B.coef = st->r_bcoef;
        B.potinfo = st->r_bpotinfo;
        B.potn = st->r_bpotn;
        B.ab2 = st->r_bab2;
        B.slot_of = st->r_slot_of;
        B.xq = st->r_xq[o];
        B.force = st->r_force;
        B.eng_cell0 = st->r_eng_cell0;
        B.eng_cdim = st->r_eng_cdim;
        B.eng_h = st->r_eng_h;
        B.capc = st->capc;
        B.ebond = st->r_ebond;
        B.acc = st->d_acc;
        B.abort = st->r_status;
        B.nengines = (int)st->engines.size();
        B.angles = st->r_angles;
        B.nangles = st->nangles;
        B.dihedrals = st->r_dihedrals;
        B.dihedral_te = st->r_dihedral_te;
        B.ndihedrals = st->ndihedrals;
        B.ab = st->r_bab;
        if (st->nbonds > 0) bond_forces<<<(st->nbonds + 127) / 128, 128, 0, st->stream>>>(B);
        if (st->nangles > 0) angle_forces<<<(st->nangles + 127) / 128, 128, 0, st->stream>>>(B);
        if (st->ndihedrals > 0) dihedral_forces<<<(st->ndihedrals + 127) / 128, 128, 0, st->stream>>>(B);
        CU(cudaGetLastError());
    }
    // One engine whose every particle is in a rigid group (rigid water): the constraint
    // kernel runs the update too (same arithmetic), one launch less per step.
    bool fuse = false;
    if (st->engines.size() == 1 && st->engines[0]->nr_rigids > 0 && st->sd_gamma <= 0.f) {
        const struct engine* e = st->engines[0];
        long long in_groups = 0;
        for (int g = 0; g < e->nr_rigids; g++) in_groups += e->rigids[g].nr_parts;
        fuse = in_groups == (long long)e->s.nr_parts;
    }
    if (!fuse) {
        const unsigned slot_blocks = (unsigned)(((size_t)st->ncells * st->capc + 255) / 256);
        integrate_cells<<<slot_blocks, 256, 0, st->stream>>>(RC, st->r_cnt[o], st->r_force, st->r_cell_engine,
                                                             st->r_engine_dt, st->r_engine_imass, st->max_type,
                                                             st->r_xq[o], st->r_v[o], st->r_status, st->d_acc,
                                                             st->r_done, st->sd_gamma, st->sd_dmax);
        CU(cudaGetLastError());
    }
    for (size_t k = 0; k < st->engines.size(); k++) {
        struct engine* e = st->engines[k];
        if (e->nr_rigids == 0) continue;
        struct rigid_resident_view view = {};
        view.fuse = fuse;
        view.force = st->r_force;
        view.imass = st->r_engine_imass + k * (size_t)st->max_type;
        view.dtf = (float)e->dt;
        view.status = st->r_status;
        view.done = st->r_done;
        view.pairs = st->d_acc + kAccPairs;
        view.slot_of = st->r_slot_of;
        view.id0 = st->id_off[k];
        view.xq = st->r_xq[o];
        view.v = st->r_v[o];
        view.capc = st->capc;
        view.cell0 = st->cell_off[k];
        view.abort = st->r_status;
        rc = rigid_eval_resident(e, &view, st->stream);
        if (rc < 0) return rc;
    }
    if (st->verlet) {                  // displacements and the next step's rebuild decision
        verlet_check<<<grid, kCellThreads, 0, st->stream>>>(RC, st->r_cnt[o], st->r_xq[o], st->r_oldx, st->d_cscale,
                                                            st->r_cell_mdx, st->r_vw, st->r_status);
        verlet_decide<<<1, 1, 0, st->stream>>>(st->r_vw, st->verlet_skin, (float)st->engines[0]->s.cutoff,
                                               st->r_status);
        CU(cudaGetLastError());
    }
    if (st->elog_cap > 0) {            // the step's energies into the log
        CU(cudaMemsetAsync(st->r_eacc, 0, sizeof(unsigned long long), st->stream));
        const unsigned slot_blocks = (unsigned)(((size_t)st->ncells * st->capc + 255) / 256);
        kinetic_cells<<<slot_blocks, 256, 0, st->stream>>>(RC, st->r_cnt[o], st->r_cell_engine, st->r_engine_imass,
                                                           st->max_type, st->r_xq[o], st->r_v[o], st->r_status,
                                                           st->r_eacc);
        energy_record<<<1, 1024, 0, st->stream>>>(st->d_cell_epot, st->ncells, st->r_ebond,
                                                  res_bonded(st) ? 3 * (int)st->engines.size() : 0, st->r_eacc,
                                                  st->r_eacc + 1, st->r_done, st->r_status, st->r_elog,
                                                  st->elog_cap);
        CU(cudaGetLastError());
    }
    return record_event(st, st->ev1);
}

// Everything a captured resident step depends on besides the device buffers' contents.
long long res_key(const NbState* st) {
    long long k = st->capc;
    k = k * 131 + st->buf_gen;
    k = k * 17 + st->warps;
    k = k * 17 + st->window;
    k = k * 3 + st->layout;
    k = k * 3 + st->stages;
    k = k * 3 + (st->occupancy == 640 ? 0 : st->occupancy == 768 ? 1 : 2);
    k = k * 3 + st->plain;
    k = k * 3 + st->record_clock;
    k = k * 2 + st->fp32acc;
    k = k * 2 + (st->sd_gamma > 0.f);
    k = k * 2 + (st->elog_cap > 0);
    k = k * 2 + st->verlet;
    return k;
}

// Issues nsteps resident steps (no host synchronisation).  Steps run as direct launches
// until every engine with rigid groups is past the P-SHAKE refinement steps; then, with
// graphs enabled, the first step from each side sets up, the second is captured, later
// ones replay.
int res_issue_steps(NbState* st, int nsteps) {
    for (int k = 0; k < nsteps; k++) {
        bool refine = false;
        for (struct engine* e : st->engines) {
            e->time += 1;
            refine = refine || (e->nr_rigids > 0 && e->time < engine_pshake_steps);
        }
        const int side = st->rside;
        const long long key = res_key(st);
        if (!st->use_graph || refine) {
            const int rc = res_issue_step(st);
            if (rc < 0) return rc;
        } else if (st->rgraph_exec[side] != nullptr && st->rgraph_key[side] == key) {
            CU(cudaGraphLaunch(st->rgraph_exec[side], st->stream));
        } else if (st->rprepared[side] != key) {
            const int rc = res_issue_step(st);
            if (rc < 0) return rc;
            st->rprepared[side] = key;
        } else {
            if (st->rgraph_exec[side]) cudaGraphExecDestroy(st->rgraph_exec[side]);
            if (st->rgraph[side]) cudaGraphDestroy(st->rgraph[side]);
            st->rgraph_exec[side] = nullptr;
            st->rgraph[side] = nullptr;
            CU(cudaStreamBeginCapture(st->stream, cudaStreamCaptureModeThreadLocal));
            st->capturing = true;
            const int rc = res_issue_step(st);
            st->capturing = false;
            cudaGraph_t g = nullptr;
            const cudaError_t end = cudaStreamEndCapture(st->stream, &g);
            if (rc < 0) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            CU(end);
            st->rgraph[side] = g;
            CU(cudaGraphInstantiate(&st->rgraph_exec[side], g, 0));
            st->rgraph_key[side] = key;
            CU(cudaGraphLaunch(st->rgraph_exec[side], st->stream));
        }
        st->rside = 1 - side;
    }
    return 0;
}

int st_resident_sync(NbState* st);

// nsteps device-resident time steps (e->time advances by nsteps).
int st_resident_steps(NbState* st, int nsteps) {
    if (!st->res_active) {
        errs_register(engine_err_cuda, "No device-resident particles (engine_cuda_resident_begin).", __LINE__,
                      __func__, __FILE__);
        return engine_err = engine_err_cuda;
    }
    CU(cudaSetDevice(st->device));
    // A step that overflowed a cell block (or the leaver lists) was aborted with every step
    // after it: the device still holds the last completed step.  Re-block with twice the
    // room from there and run the remaining steps (at most 8 times per call).
    int left = nsteps, regrows = 0;
    st->res_dirty = st->res_dirty || nsteps > 0;
    while (left > 0) {
        const int side0 = st->rside;
        int rc = res_issue_steps(st, left);
        if (rc < 0) return rc;
        unsigned long long w[3] = {0, 0, 0};
        CU(cudaMemcpyAsync(&w[0], st->r_status, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st->stream));
        CU(cudaMemcpyAsync(&w[1], st->r_done, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st->stream));
        CU(cudaStreamSynchronize(st->stream));
        const long long completed = (long long)w[1] - st->res_done;
        st->res_done = (long long)w[1];
        st->res_pairs = (long long)w[2];
        if (w[0] == 0) break;
        for (struct engine* e : st->engines) e->time -= (int)(left - completed);
        st->rside = side0 ^ (int)(completed & 1);
        left -= (int)completed;
        const bool cells = (w[0] & kStatusResidentOverflow) != 0, movers = (w[0] & kStatusMoverOverflow) != 0;
        if (w[0] & kStatusNonFinite) {
            errs_register(engine_err_cuda, "Non-finite particle position or velocity.", __LINE__, __func__, __FILE__);
            return engine_err = engine_err_cuda;
        }
        if (++regrows > 8 || (cells && st->capc >= kMaxPartsPerCell)) {
            errs_register(engine_err_maxparts, "Max. number of parts per cell exceeded during resident steps.",
                          __LINE__, __func__, __FILE__);
            return engine_err = engine_err_maxparts;
        }
        // the abort word has served: the side it protected is the one to bring back
        CU(cudaMemsetAsync(st->r_status, 0, sizeof(unsigned long long), st->stream));
        rc = st_resident_sync(st);
        if (rc < 0) return rc;
        const long long done = st->res_done_total + st->res_done;
        const long long pairs = st->res_pairs_total + st->res_pairs;
        const int total_regrows = st->res_regrows + 1;
        rc = st_resident_begin(st, cells ? 2 * st->res_margin : st->res_margin, movers ? 2 * st->mcap : st->mcap);
        if (rc < 0) return rc;
        st->res_done_total = done;
        st->res_pairs_total = pairs;
        st->res_regrows = total_regrows;
        if (st->elog_cap > 0) {       // the log keeps counting from the steps already done
            const unsigned long long base = (unsigned long long)done;
            CU(cudaMemcpy(st->r_eacc + 1, &base, sizeof(base), cudaMemcpyHostToDevice));
        }
    }
    return 0;
}

// The download of the current side, queued on the state's stream: cell offsets by a scan
// of the counts, the particles compacted in cell order; down: the status and completed-
// step words and the counts first, then the particles in chunks with an event after each,
// then energies, counters and constraint statistics.
int res_download_issue(NbState* st) {
    const int nc = st->ncells, ne = (int)st->engines.size(), side = st->rside;
    const size_t np = (size_t)st->res_nparts;
    const ResidentCells RC = res_cells(st);
    const int nb = (nc + kScanBlock - 1) / kScanBlock;
    const int K = res_chunks(st, np);
    int rc = chunk_events(st, K + 1);
    if (rc < 0) return rc;
    if (nc > 0) {
        scan_counts_sums<<<nb, kScanBlock, 0, st->stream>>>(st->r_cnt[side], nc, st->capc, st->r_bsum);
        scan_counts_blocks<<<1, kScanBlock, 0, st->stream>>>(st->r_bsum, nb);
        scan_counts_apply<<<nb, kScanBlock, 0, st->stream>>>(st->r_cnt[side], nc, st->capc, st->r_bsum, st->r_doff);
        compact_cells<<<res_grid(st), kCellThreads, 0, st->stream>>>(RC, st->r_xq[side], st->r_v[side],
                                                                     st->r_pid[side], st->r_cnt[side], st->r_doff,
                                                                     st->r_force, np, st->r_up_of, st->r_dense,
                                                                     reinterpret_cast<float*>(st->r_dense + np),
                                                                     reinterpret_cast<float*>(st->r_dense + np) + 3 * np);
        CU(cudaGetLastError());
    }
    CU(cudaMemcpyAsync(st->h_words, st->r_status, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st->stream));
    CU(cudaMemcpyAsync(st->h_words + 1, st->r_done, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       st->stream));
    CU(cudaMemcpyAsync(st->h_rcount, st->r_cnt[side], sizeof(int) * nc, cudaMemcpyDeviceToHost, st->stream));
    // the cells' energies and virials ahead of the particles: the host sets each cell's
    // energy while it rebuilds the cell
    CU(cudaMemcpyAsync(st->h_cell_epot, st->d_cell_epot, sizeof(unsigned long long) * 2 * st->ncells,
                       cudaMemcpyDeviceToHost, st->stream));
    CU(cudaEventRecord(st->chunk_ev[0], st->stream));
    const float* dv3 = reinterpret_cast<const float*>(st->r_dense + np);
    float* hv3 = reinterpret_cast<float*>(st->h_dense + np);
    for (int k = 0; k < K; k++) {
        const size_t q0 = np * k / K, q1 = np * (k + 1) / K;
        CU(cudaMemcpyAsync(st->h_dense + q0, st->r_dense + q0, sizeof(float4) * (q1 - q0), cudaMemcpyDeviceToHost,
                           st->stream));
        for (int a = 0; a < 2; a++)          // velocities, forces
            CU(cudaMemcpyAsync(hv3 + 3 * (a * np + q0), dv3 + 3 * (a * np + q0), 3 * sizeof(float) * (q1 - q0),
                               cudaMemcpyDeviceToHost, st->stream));
        CU(cudaEventRecord(st->chunk_ev[k + 1], st->stream));
    }
    CU(cudaMemcpyAsync(st->h_acc, st->d_acc, sizeof(unsigned long long) * kAccCount, cudaMemcpyDeviceToHost,
                       st->stream));
    if (res_bonded(st))
        CU(cudaMemcpyAsync(st->h_ebond, st->r_ebond, sizeof(unsigned long long) * 3 * ne, cudaMemcpyDeviceToHost,
                           st->stream));
    for (struct engine* e : st->engines)
        if (e->nr_rigids > 0) rigid_resident_stats(e, st->stream, 0);
    return 0;
}

// Waits for the download queued by res_download_issue and rebuilds the host cells from it,
// chunk by chunk as the copies land; energies and statistics.  *status: the device status
// word (nonzero: the step was aborted and the host cells are unchanged).
int res_download_finish(NbState* st, unsigned long long* status) {
    const int nc = st->ncells, ne = (int)st->engines.size();
    const size_t np = (size_t)st->res_nparts;
    const int K = res_chunks(st, np);
    CU(cudaEventSynchronize(st->chunk_ev[0]));
    *status = st->h_words[0];
    if (*status != 0) {
        CU(cudaStreamSynchronize(st->stream));
        return 0;
    }
    int* cnt = st->h_rcount;                     // counts, then offsets
    int* off = st->h_rcount + nc + 1;
    // Every particle must still be in one of its engine's cells; else the host keeps its copy.
    off[0] = 0;
    for (int c = 0; c < nc; c++) off[c + 1] = off[c] + std::min(cnt[c], st->capc);
    for (int k = 0; k < ne; k++)
        if (off[st->cell_off[k + 1]] - off[st->cell_off[k]] != st->res_engine_n[k]) {
            CU(cudaStreamSynchronize(st->stream));
            errs_register(engine_err_maxparts, "Particles missing from the device cells.", __LINE__, __func__,
                          __FILE__);
            return engine_err = engine_err_maxparts;
        }
    // The host cells take the device's particles in the device's order (id, charge and
    // flags of each particle from the upload).
    std::atomic<int> fail(0);
    double t_rebuild = 0.0;
    int cdone = 0;
    const float* hv3 = reinterpret_cast<const float*>(st->h_dense + np);
    const float* hf3 = hv3 + 3 * np;
    // Each cell's energy is set by the thread that rebuilds the cell; the engines' energy
    // and virial sums per host thread (own 64-byte lines), summed afterwards (integers).
    const unsigned long long* cep = st->h_cell_epot;
    const unsigned long long* cvir = st->h_cell_epot + nc;
    const int nparts = HostPool::get().threads();
    const size_t stride = ((size_t)2 * ne + 7) & ~(size_t)7;
    std::vector<long long> psum((size_t)nparts * stride, 0);
    for (int k = 0; k < K; k++) {
        const int pend = (int)(np * (k + 1) / K);
        const int cend = k == K - 1 ? nc : (int)(std::upper_bound(off + 1, off + nc + 1, pend) - (off + 1));
        CU(cudaEventSynchronize(st->chunk_ev[k + 1]));
        const double t0 = now_ms();
        const int c0 = cdone;
        HostPool::get().run(cend - c0, cell_grain(st), [&](int part, int rb, int re) {
            const int cb = c0 + rb, ce = c0 + re;
            long long* my = psum.data() + (size_t)part * stride;
            for (int c = cb; c < ce; c++) {
                if (c + 8 < ce) __builtin_prefetch(st->flat_cells[c + 8], 1);
                if (c + 4 < ce) __builtin_prefetch(st->flat_cells[c + 4]->parts, 1);
                const size_t ke =
                    std::upper_bound(st->cell_off.begin(), st->cell_off.end(), c) - st->cell_off.begin() - 1;
                const int lo = st->id_off[ke];
                struct space* sp = &st->engines[ke]->s;
                struct cell* cl = st->flat_cells[c];
                const int n = off[c + 1] - off[c];
                const long long ev = (long long)cep[c];
                my[2 * ke] += ev;
                my[2 * ke + 1] += (long long)cvir[c];
                cl->epot = (double)ev / kEnergyScale;
                if (n > cl->size) {             // the old contents are replaced, not copied
                    const int nsize = std::max(n, std::max(2 * cl->size, 16));
                    struct part* fresh = nullptr;
                    if (posix_memalign(reinterpret_cast<void**>(&fresh), 64, sizeof(struct part) * nsize) != 0) {
                        fail = 1;
                        return;
                    }
                    free(cl->parts);
                    cl->parts = fresh;
                    cl->size = nsize;
                }
                for (int q = 0; q < n; q++) {
                    const size_t o = (size_t)off[c] + q;
                    const float4 x = st->h_dense[o];
                    int ou;                                  // the particle's upload index
                    std::memcpy(&ou, &x.w, sizeof(int));
                    if (ou < 0 || (size_t)ou >= np) {
                        fail = 2;
                        return;
                    }
                    const NbState::UpAux& ax = st->up_aux[ou];
                    const float* v = hv3 + 3 * o;
                    const float* f = hf3 + 3 * o;
                    struct part t;
                    t.x[0] = x.x; t.x[1] = x.y; t.x[2] = x.z; t.x[3] = 0.f;
                    t.v[0] = v[0]; t.v[1] = v[1]; t.v[2] = v[2]; t.v[3] = 0.f;
                    t.f[0] = f[0]; t.f[1] = f[1]; t.f[2] = f[2]; t.f[3] = 0.f;
                    t.q = ax.q;
                    t.id = ax.gid - lo;
                    t.vid = ax.vid;
                    t.type = ax.type;
                    t.flags = ax.flags;
                    struct part* p = &cl->parts[q];
                    *p = t;
                    // space_relink, inline; most particles keep their slot from one step to
                    // the next, and an unchanged entry is not written (no dirty line)
                    if (sp->partlist[t.id] != p) sp->partlist[t.id] = p;
                    if (sp->celllist[t.id] != cl) sp->celllist[t.id] = cl;
                }
                cl->count = n;
            }
            const size_t q0 = (size_t)off[cb], q1 = (size_t)off[ce];
            evict_lines(st->h_dense + q0, sizeof(float4) * (q1 - q0));
            for (int a = 0; a < 2; a++) evict_lines(hv3 + 3 * (a * np + q0), 3 * sizeof(float) * (q1 - q0));
        });
        t_rebuild += now_ms() - t0;
        cdone = cend;
    }
    st->bstats.ms_unpack = (float)t_rebuild;
    CU(cudaStreamSynchronize(st->stream));
    if (fail == 2) {
        errs_register(engine_err_cuda, "A downloaded particle has no upload index.", __LINE__, __func__, __FILE__);
        return engine_err = engine_err_cuda;
    }
    if (fail) {
        errs_register(engine_err_malloc, "Could not grow a host cell.", __LINE__, __func__, __FILE__);
        return engine_err = engine_err_malloc;
    }
    for (int k = 0; k < ne; k++) {
        struct space* sp = &st->engines[k]->s;
        sp->epot = sp->epot_nonbond = sp->epot_bond = sp->epot_angle = sp->epot_dihedral = sp->epot_exclusion = 0.0;
    }
    st->res_dirty = false;
    std::vector<long long> sums((size_t)2 * ne, 0);
    for (int q = 0; q < nparts; q++)
        for (int k = 0; k < 2 * ne; k++) sums[k] += psum[(size_t)q * stride + k];
    const int rc = finish_stats(st, &sums);
    for (int k = 0; k < ne; k++) {
        struct space* sp = &st->engines[k]->s;
        if (res_bonded(st)) {
            sp->epot_bond = (double)(long long)st->h_ebond[k] / kEnergyScale;
            sp->epot_angle = (double)(long long)st->h_ebond[ne + k] / kEnergyScale;
            sp->epot_dihedral = (double)(long long)st->h_ebond[2 * ne + k] / kEnergyScale;
        }
        sp->epot += sp->epot_nonbond + sp->epot_bond + sp->epot_angle + sp->epot_dihedral;
    }
    return rc;
}

// Downloads the current side into the host cells, each chunk's cells rebuilt on the host
// threads while the next one copies.  *status receives the abort word; when it is set
// nothing is rebuilt (the host cells keep what they held).
int res_download(NbState* st, unsigned long long* status) {
    const int rc = res_download_issue(st);
    if (rc < 0) return rc;
    return res_download_finish(st, status);
}

// Brings the engines' host cells up to date: positions, velocities and the last
// evaluation's forces of every particle, in the device's cell order, energies and
// statistics of the last step.
int st_resident_sync(NbState* st) {
    if (!st->res_active) {
        errs_register(engine_err_cuda, "No device-resident particles (engine_cuda_resident_begin).", __LINE__,
                      __func__, __FILE__);
        return engine_err = engine_err_cuda;
    }
    CU(cudaSetDevice(st->device));
    unsigned long long status = 0;
    const int rc = res_download(st, &status);
    if (rc < 0) return rc;
    if (status != 0) {
        errs_register(engine_err_maxparts, "Device cell capacity exceeded during resident steps.", __LINE__,
                      __func__, __FILE__);
        return engine_err = engine_err_maxparts;
    }
    return 0;
}

}  // namespace

// ---------------------------------------------------------------- single engine

extern "C" void nb_parallel_for(int n, int grain, void (*fn)(void*, int, int, int), void* ctx) {
    HostPool::get().run(n, grain, [&](int part, int b, int e) { fn(ctx, part, b, e); });
}

extern "C" int nb_host_parts(void) { return HostPool::get().threads(); }

extern "C" void nb_zero_cells(struct space* s) {
    const int grain = (int)std::max(16LL, host_grain_parts() / (s->nr_parts / std::max(1, s->nr_cells) + 1));
    HostPool::get().run(s->nr_cells, grain, [&](int, int b, int e) {
        for (int c = b; c < e; c++) {
            struct cell* cl = &s->cells[c];
            cl->epot = 0.0;
            for (int q = 0; q < cl->count; q++) cl->parts[q].f[0] = cl->parts[q].f[1] = cl->parts[q].f[2] = 0.0f;
        }
    });
}

extern "C" void* nb_engine_stream(struct engine* e) {
    return (e != nullptr && e->cuda != nullptr) ? static_cast<void*>(state(e)->stream) : nullptr;
}

extern "C" int nb_device_free(struct engine* e) {
    if (e == nullptr || e->cuda == nullptr) return 0;
    state_free(state(e));
    e->cuda = nullptr;
    return 0;
}

extern "C" int engine_cuda_setdevice(struct engine* e, int id) {
    if (e == nullptr) return engine_err_null;
    int n = 0;
    CU(cudaGetDeviceCount(&n));
    if (id < 0 || id >= n) {
        errs_register(engine_err_range, "No such CUDA device.", __LINE__, __func__, __FILE__);
        return engine_err = engine_err_range;
    }
    e->device = id;
    return 0;
}

extern "C" int engine_cuda_setdevices(struct engine* e, int nr_devices, int* ids) {
    if (e == nullptr || ids == nullptr) return engine_err_null;
    if (nr_devices != 1) {
        errs_register(engine_err_nyi, "Only one device per engine.", __LINE__, __func__, __FILE__);
        return engine_err = engine_err_nyi;
    }
    return engine_cuda_setdevice(e, ids[0]);
}

extern "C" int engine_cuda_settune(struct engine* e, int warps, int plain) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    return st_settune(state(e), warps, plain);
}

extern "C" int engine_cuda_setwindow(struct engine* e, int window) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    if (window != 4 && window != 8) return engine_err_range;
    state(e)->window = window;
    return 0;
}

static int st_setlayout(NbState* st, int layout, int stages, int occupancy) {
    if ((layout != 0 && layout != 1) || (stages != 1 && stages != 2) ||
        (occupancy != 640 && occupancy != 768 && occupancy != 1024) || (stages == 2 && occupancy == 768))
        return engine_err_range;
    st->layout = layout;
    st->stages = stages;
    st->occupancy = occupancy;
    return 0;
}

extern "C" int engine_cuda_setlayout(struct engine* e, int layout, int stages, int occupancy) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    return st_setlayout(state(e), layout, stages, occupancy);
}

// Rebuilds (re-binning + sort) of the resident steps since the last upload, with
// engine_flag_verlet; -1 without the flag or resident particles.
extern "C" int engine_cuda_verlet_rebuilds(struct engine* e, int* rebuilds) {
    if (e == nullptr || e->cuda == nullptr || rebuilds == nullptr) return engine_err_null;
    NbState* st = state(e);
    *rebuilds = -1;
    if (!st->res_active || !st->verlet) return 0;
    CU(cudaSetDevice(st->device));
    CU(cudaStreamSynchronize(st->stream));
    int w[4];
    CU(cudaMemcpy(w, st->r_vw, sizeof(w), cudaMemcpyDeviceToHost));
    *rebuilds = w[2];
    return 0;
}

// FP32 force accumulation (fp32 = 1: the plain form adds each task's partial forces as
// floats with float atomics) or 64-bit fixed point (0, the default).
// Polls per bounded wait of the sweeps on the engine's device (polls <= 0: the default,
// kSpinLimit).  A wait that runs out makes the evaluation report a copy timeout.
extern "C" int engine_cuda_setspin(struct engine* e, int polls) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    NbState* st = state(e);
    const int v = polls > 0 ? polls : kSpinLimit;
    CU(cudaSetDevice(st->device));
    CU(cudaStreamSynchronize(st->stream));
    CU(cudaMemcpyToSymbol(c_spin_limit, &v, sizeof(v)));
    return 0;
}

// Test hook of the failure path: with enable = 1 the sweeps on the engine's device neither
// arrive on their staging mbarriers nor issue a copy, so every wait runs out after the spin
// limit, the evaluation fails with engine_err_cuda ("Bulk copy into shared memory timed
// out.") and nothing is in flight; 0 restores normal copies.
extern "C" int engine_cuda_copytimeout_test(struct engine* e, int enable) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    if (enable != 0 && enable != 1) return engine_err_range;
    NbState* st = state(e);
    CU(cudaSetDevice(st->device));
    CU(cudaStreamSynchronize(st->stream));
    CU(cudaMemcpyToSymbol(c_skip_copies, &enable, sizeof(enable)));
    return 0;
}

extern "C" int engine_cuda_setaccum(struct engine* e, int fp32) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    if (fp32 != 0 && fp32 != 1) return engine_err_range;
    state(e)->fp32acc = fp32;
    return 0;
}

// Steepest-descent resident steps: x += g f, |g f| <= dmax, v = 0 (gamma <= 0: time steps).
extern "C" int engine_cuda_minimize(struct engine* e, double gamma, double dmax) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    if (gamma > 0.0 && !(dmax > 0.0)) return engine_err_range;
    NbState* st = state(e);
    st->sd_gamma = gamma > 0.0 ? (float)gamma : 0.f;
    st->sd_dmax = gamma > 0.0 ? (float)dmax : 0.f;
    return 0;
}

// Per-step energy log of the resident steps: a ring of `cap` records (0: off).  Setting it
// (again) clears the log.
extern "C" int engine_cuda_energylog(struct engine* e, int cap) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    if (cap < 0) return engine_err_range;
    NbState* st = state(e);
    CU(cudaSetDevice(st->device));
    CU(cudaStreamSynchronize(st->stream));
    if (cap != st->elog_cap) {
        if (st->r_elog) CU(cudaFree(st->r_elog));
        if (st->r_eacc) CU(cudaFree(st->r_eacc));
        st->r_elog = nullptr;
        st->r_eacc = nullptr;
        st->elog_cap = 0;
        st->buf_gen++;
        if (cap > 0) {
            CU(cudaMalloc(&st->r_elog, sizeof(unsigned long long) * 4 * (size_t)cap));
            CU(cudaMalloc(&st->r_eacc, sizeof(unsigned long long) * 2));
        }
        st->elog_cap = cap;
    }
    if (cap > 0) {
        CU(cudaMemset(st->r_elog, 0, sizeof(unsigned long long) * 4 * (size_t)cap));
        const unsigned long long base =
            st->res_active ? (unsigned long long)(st->res_done_total + st->res_done) : 0ull;
        CU(cudaMemcpy(st->r_eacc + 1, &base, sizeof(base), cudaMemcpyHostToDevice));
    }
    return 0;
}

// The records of the log in step order: out[4 k + 0..3] = resident step number (1 = the
// first step after engine_cuda_resident_begin), potential energy (nonbonded + bonded),
// kinetic energy of the velocities after the step, their sum (kJ/mol).  Returns the count.
extern "C" int engine_cuda_energylog_read(struct engine* e, double* out, int max) {
    if (e == nullptr || e->cuda == nullptr || (out == nullptr && max > 0)) return engine_err_null;
    NbState* st = state(e);
    if (st->elog_cap <= 0) return 0;
    CU(cudaSetDevice(st->device));
    CU(cudaStreamSynchronize(st->stream));
    std::vector<unsigned long long> h(4 * (size_t)st->elog_cap);
    CU(cudaMemcpy(h.data(), st->r_elog, sizeof(unsigned long long) * h.size(), cudaMemcpyDeviceToHost));
    std::vector<int> idx;
    for (int k = 0; k < st->elog_cap; k++)
        if (h[4 * (size_t)k] != 0) idx.push_back(k);
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return h[4 * (size_t)a] < h[4 * (size_t)b]; });
    const int n = std::min((int)idx.size(), std::max(max, 0));
    const size_t skip = idx.size() - (size_t)n;      // the latest records when max is smaller
    for (int q = 0; q < n; q++) {
        const unsigned long long* r = &h[4 * (size_t)idx[skip + q]];
        const double ep = (double)(long long)r[1] / kEnergyScale, ek = (double)(long long)r[2] / kEnergyScale;
        out[4 * q + 0] = (double)r[0];
        out[4 * q + 1] = ep;
        out[4 * q + 2] = ek;
        out[4 * q + 3] = ep + ek;
    }
    return n;
}

extern "C" int engine_cuda_graph(struct engine* e, int enable) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    NbState* st = state(e);
    st->use_graph = enable != 0;
    if (!st->use_graph) drop_graph(st);
    st->prepared_key = -1;
    return 0;
}

extern "C" int engine_cuda_autotune(struct engine* e, int reps, int* warps, int* layout, int* stages, int* occupancy,
                                    float* ms) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    return st_autotune(state(e), reps, warps, layout, stages, occupancy, ms);
}

extern "C" int engine_cuda_load(struct engine* e) {
    if (e == nullptr) return engine_err_null;
    if (e->cuda) nb_device_free(e);
    NbState* st = new NbState();
    e->cuda = st;
    st->engines.assign(1, e);
    return load_state(st);
}

extern "C" int engine_cuda_load_parts(struct engine* e) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    return st_load_parts(state(e));
}

extern "C" int engine_cuda_unload_parts(struct engine* e) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    return st_unload_parts(state(e));
}

extern "C" int engine_nonbond_cuda(struct engine* e) {
    if (e == nullptr) return engine_err_null;
    if (e->cuda == nullptr && engine_cuda_load(e) < 0) return engine_err_cuda;
    return st_nonbond(state(e));
}

// engine_zero_forces + engine_nonbond_cuda in one pass over the particles.
extern "C" int engine_nonbond_cuda_fresh(struct engine* e) {
    if (e == nullptr) return engine_err_null;
    if (e->cuda == nullptr && engine_cuda_load(e) < 0) return engine_err_cuda;
    return st_nonbond(state(e), true);
}

// Sort + sweep on the particles already resident on the device (no host copies, no
// synchronisation); results stay on the device until engine_cuda_unload_parts.
extern "C" int engine_nonbond_cuda_resident(struct engine* e) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    return st_resident(state(e));
}

// Runs further launches on a caller-provided stream (e.g. the framework's current stream).
extern "C" int engine_cuda_resident_begin(struct engine* e, int margin) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    const int rc = st_resident_begin(state(e), margin, 16);
    return rc < 0 ? rc : elog_restart(state(e));
}

extern "C" int engine_cuda_resident_steps(struct engine* e, int nsteps) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    return st_resident_steps(state(e), nsteps);
}

extern "C" int engine_cuda_resident_sync(struct engine* e) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    return st_resident_sync(state(e));
}

int st_resident_info(const NbState* st, int* capc, int* mcap, long long* steps, long long* pairs, int* regrows) {
    if (!st->res_active) {
        errs_register(engine_err_cuda, "No device-resident particles (engine_cuda_resident_begin).", __LINE__,
                      __func__, __FILE__);
        return engine_err = engine_err_cuda;
    }
    if (capc) *capc = st->capc;
    if (mcap) *mcap = st->mcap;
    if (steps) *steps = st->res_done_total + st->res_done;
    if (pairs) *pairs = st->res_pairs_total + st->res_pairs;
    if (regrows) *regrows = st->res_regrows;
    return 0;
}

// One engine_step of every engine on the device with the host cells as input and output:
// the particles go up, one resident step runs (re-binning, sort, sweep, integration, rigid
// constraints), the particles, forces, energies and statistics come back, with a single
// host synchronisation.  The device blocks are kept between calls and re-made only when a
// cell has outgrown them (before the step, or when the step itself overflowed and was
// aborted: the host copy is then unchanged and the step runs again in larger blocks).  If
// resident steps left the device ahead of the host, the step continues from the device.
int st_step_device(NbState* st) {
    CU(cudaSetDevice(st->device));
    const double t0 = now_ms();
    st->bstats.ms_pack = st->bstats.ms_unpack = 0.f;
    int rc = 0;
    if (st->res_active && st->res_dirty) {
        rc = st_resident_sync(st);
        if (rc < 0) return rc;
    }
    int margin = 8, mcap = st->res_active ? st->mcap : 16;
    for (int attempt = 0;; attempt++) {
        long long n = 0;
        const int maxc = res_host_counts(st, &n);
        if (st->res_active && n == st->res_nparts && maxc + 4 <= st->capc && st->mcap >= mcap &&
            st->bonds_key == res_bonds_key(st)) {
            rc = res_upload(st);
        } else {
            rc = st_resident_begin(st, margin, mcap);
        }
        if (rc < 0) return rc;
        rc = res_issue_steps(st, 1);
        if (rc < 0) return rc;
        unsigned long long status = 0;
        rc = res_download(st, &status);
        if (rc < 0) return rc;
        if (status == 0) {
            st->res_done = (long long)st->h_words[1];
            st->res_pairs = (long long)st->h_words[2];
            break;
        }
        if (status & kStatusNonFinite) {
            errs_register(engine_err_cuda, "Non-finite particle position or velocity.", __LINE__, __func__, __FILE__);
            return engine_err = engine_err_cuda;
        }
        // Aborted on the device: the host cells still hold the step's input.
        for (struct engine* e : st->engines) e->time -= 1;
        const bool cells = (status & kStatusResidentOverflow) != 0;
        if (attempt >= 8 || (cells && st->capc >= kMaxPartsPerCell)) {
            errs_register(engine_err_maxparts, "Max. number of parts per cell exceeded.", __LINE__, __func__,
                          __FILE__);
            return engine_err = engine_err_maxparts;
        }
        margin = cells ? 2 * std::max(st->res_margin, 8) : st->res_margin;
        if (status & kStatusMoverOverflow) mcap = 2 * st->mcap;
        res_free(st);
    }
    st->bstats.ms_device = (float)(now_ms() - t0) - st->bstats.ms_pack - st->bstats.ms_unpack;
    share_times(st);
    return rc;
}

// ---- engine_step of a batch in groups of engines
//
// The host packs a group's cells and queues its upload, step and download on the group's
// stream, then packs the next group while the device works; afterwards it rebuilds each
// group's cells as its download lands, while the later groups' downloads still run.  Each
// group is a batch of its own (own device blocks, graphs and stream), so the step is the
// same per engine as in one batch.

namespace {

// Groups of a batch's engine_step: as requested, else one per 2^18 particles (at most 4);
// never more than the engines.  A batch that holds resident particles steps as one group.
int step_groups(const NbState* st) {
    if (st->res_active) return 1;
    long long n = 0;
    for (const struct cell* c : st->flat_cells) n += c->count;
    const long long k = st->groups_req > 0 ? st->groups_req : std::min(4LL, std::max(1LL, n >> 18));
    return (int)std::max(1LL, std::min(k, (long long)st->engines.size()));
}

// The batch's launch shape and step options, for a group.
void copy_shape(NbState* c, const NbState* st) {
    c->warps = st->warps;
    c->window = st->window;
    c->layout = st->layout;
    c->stages = st->stages;
    c->occupancy = st->occupancy;
    c->use_graph = st->use_graph;
    c->plain = st->plain;
    c->fp32acc = st->fp32acc;
    c->sd_gamma = st->sd_gamma;
    c->sd_dmax = st->sd_dmax;
    c->max_chunks = std::max(1, 8 / (int)st->groups.size());
    c->tiny_inherited = tiny_tasks_of(st);       // the same sweep path as the whole batch
}

// (Re)builds k group states over contiguous runs of engines of about equal particle counts.
int make_groups(NbState* st, int k) {
    for (NbState* g : st->groups) state_free(g);
    st->groups.clear();
    const size_t ne = st->engines.size();
    std::vector<long long> cum(ne + 1, 0);
    for (size_t i = 0; i < ne; i++) {
        long long n = 0;
        const struct space* sp = &st->engines[i]->s;
        for (int c = 0; c < sp->nr_cells; c++) n += sp->cells[c].count;
        cum[i + 1] = cum[i] + n;
    }
    size_t e0 = 0;
    for (int g = 0; g < k; g++) {
        size_t e1 = ne;
        if (g < k - 1) {
            e1 = (size_t)(std::lower_bound(cum.begin(), cum.end(), cum[ne] * (g + 1) / k) - cum.begin());
            e1 = std::min(std::max(e1, e0 + 1), ne - (size_t)(k - 1 - g));
        }
        NbState* c = new NbState();
        c->engines.assign(st->engines.begin() + e0, st->engines.begin() + e1);
        const int rc = load_state(c);
        if (rc < 0) {
            state_free(c);
            return rc;
        }
        st->groups.push_back(c);
        e0 = e1;
    }
    return 0;
}

int st_step_grouped(NbState* st, int k) {
    CU(cudaSetDevice(st->device));
    const double t0 = now_ms();
    if ((int)st->groups.size() != k) {
        const int rc = make_groups(st, k);
        if (rc < 0) return rc;
    }
    CU(cudaStreamSynchronize(st->stream));       // work the caller queued on the batch's stream
    double pack = 0.0, unpack = 0.0;
    std::vector<char> begun(k, 0);
    // On an error the groups already queued are still finished (their host cells rebuilt),
    // no further group is started, and the first error is returned.
    int err = 0;
    for (int g = 0; g < k && err == 0; g++) {
        NbState* c = st->groups[g];
        copy_shape(c, st);
        long long n = 0;
        const int maxc = res_host_counts(c, &n);
        if (!(c->res_active && n == c->res_nparts && maxc + 4 <= c->capc && c->bonds_key == res_bonds_key(c)))
            continue;                            // new or outgrown blocks: stepped on their own below
        int rc = res_upload(c);
        if (rc == 0) {
            pack += c->bstats.ms_pack;
            rc = res_issue_steps(c, 1);
        }
        if (rc == 0) rc = res_download_issue(c);
        if (rc < 0) {
            CU(cudaStreamSynchronize(c->stream));
            err = rc;
            break;
        }
        begun[g] = 1;
    }
    struct nb_stats tot = {};
    for (int g = 0; g < k; g++) {
        NbState* c = st->groups[g];
        unsigned long long status = 1;
        if (begun[g]) {
            const int rc = res_download_finish(c, &status);
            unpack += c->bstats.ms_unpack;
            if (rc < 0) {
                if (err == 0) err = rc;
                continue;
            }
        }
        if (err != 0) continue;
        if (status == 0) {
            c->res_done = (long long)c->h_words[1];
            c->res_pairs = (long long)c->h_words[2];
        } else {
            // aborted on the device (the host cells still hold the input), or not begun
            if (begun[g])
                for (struct engine* e : c->engines) e->time -= 1;
            const int rc = st_step_device(c);
            if (rc < 0) {
                err = rc;
                continue;
            }
            pack += c->bstats.ms_pack;
            unpack += c->bstats.ms_unpack;
        }
        tot.epot += c->bstats.epot;
        tot.virial += c->bstats.virial;
        tot.pairs += c->bstats.pairs;
        tot.excluded += c->bstats.excluded;
        tot.candidates += c->bstats.candidates;
        tot.status |= c->bstats.status;
    }
    if (err != 0) return err;
    st->bstats.epot = tot.epot;
    st->bstats.virial = tot.virial;
    st->bstats.pairs = tot.pairs;
    st->bstats.excluded = tot.excluded;
    st->bstats.candidates = tot.candidates;
    st->bstats.status = tot.status;
    if (st->engines.size() > 1)                  // counts are kept for the batch only
        for (struct engine* e : st->engines) e->stats.pairs = e->stats.excluded = e->stats.candidates = -1;
    st->bstats.ms_pack = (float)pack;
    st->bstats.ms_unpack = (float)unpack;
    st->bstats.ms_device = (float)(now_ms() - t0 - pack - unpack);
    share_times(st);
    return 0;
}

}  // namespace

extern "C" int engine_cuda_step(struct engine* e) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    return st_step_device(state(e));
}

extern "C" int engine_cuda_resident_info(struct engine* e, int* capc, int* mcap, long long* steps, long long* pairs,
                                         int* regrows) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    return st_resident_info(state(e), capc, mcap, steps, pairs, regrows);
}

extern "C" int engine_cuda_resident_end(struct engine* e) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    NbState* st = state(e);
    int rc = st->res_active ? st_resident_sync(st) : 0;
    res_free(st);
    return rc;
}

extern "C" int engine_cuda_setstream(struct engine* e, void* stream) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    return st_setstream(state(e), stream);
}

extern "C" int engine_cuda_getsort(struct engine* e, int cid, unsigned int* keys, int size) {
    if (e == nullptr || e->cuda == nullptr || keys == nullptr) return engine_err_null;
    NbState* st = state(e);
    struct space* s = &e->s;
    if (cid < 0 || cid >= s->nr_cells) return engine_err_range;
    int n = s->cells[cid].count, pad = (n + 3) & ~3;
    if (size < 13 * n) return engine_err_range;
    std::vector<unsigned> buf(13 * (size_t)pad + 1);
    CU(cudaStreamSynchronize(st->stream));
    CU(cudaMemcpy(buf.data(), st->d_keys + 13 * (size_t)st->h_cstart[cid], sizeof(unsigned) * 13 * (size_t)pad,
                  cudaMemcpyDeviceToHost));
    for (int sid = 0; sid < 13; sid++)
        for (int k = 0; k < n; k++) keys[sid * n + k] = buf[(size_t)sid * pad + k];
    return 0;
}

// Device times of the last evaluation: sort + sweep, and the sweep kernel alone (waits for
// the launching stream).
extern "C" int engine_cuda_kernel_times(struct engine* e, float* total_ms, float* sweep_ms) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    return st_kernel_times(state(e), total_ms, sweep_ms);
}

// ---------------------------------------------------------------- batches of engines
//
// A batch evaluates the nonbonded forces of many independent engines (replicas: same
// force field, own particles and box) with one sort launch and one persistent sweep over
// the concatenated task list, so that systems of a few thousand particles -- too small to
// fill a B200 alone -- share the GPU.  The engines keep their own host data; the batch owns
// the device state.  Energies and virials are kept per engine; pair counts for the batch.

namespace {
NbState* bstate(struct engine_batch* b) { return reinterpret_cast<NbState*>(b); }
}  // namespace

extern "C" int engine_batch_create(struct engine** engines, int n, struct engine_batch** out) {
    if (engines == nullptr || out == nullptr || n < 1) return engine_err_null;
    for (int k = 0; k < n; k++)
        if (engines[k] == nullptr) return engine_err_null;
    NbState* st = new NbState();
    st->engines.assign(engines, engines + n);
    const int rc = load_state(st);
    if (rc < 0) {
        state_free(st);
        return rc;
    }
    *out = reinterpret_cast<struct engine_batch*>(st);
    return 0;
}

extern "C" int engine_batch_free(struct engine_batch* b) {
    if (b == nullptr) return 0;
    state_free(bstate(b));
    return 0;
}

extern "C" int engine_batch_load_parts(struct engine_batch* b) {
    if (b == nullptr) return engine_err_null;
    return st_load_parts(bstate(b));
}

extern "C" int engine_batch_resident(struct engine_batch* b) {
    if (b == nullptr) return engine_err_null;
    return st_resident(bstate(b));
}

extern "C" int engine_batch_unload_parts(struct engine_batch* b) {
    if (b == nullptr) return engine_err_null;
    return st_unload_parts(bstate(b));
}

extern "C" int engine_batch_nonbond(struct engine_batch* b) {
    if (b == nullptr) return engine_err_null;
    return st_nonbond(bstate(b));
}

extern "C" int engine_batch_nonbond_fresh(struct engine_batch* b) {
    if (b == nullptr) return engine_err_null;
    return st_nonbond(bstate(b), true);
}

// One time step of every engine: re-binning, force evaluation in one batch, symplectic
// Euler update (engine_step for each engine, with the forces computed together).
extern "C" int engine_batch_step(struct engine_batch* b) {
    if (b == nullptr) return engine_err_null;
    NbState* st = bstate(b);
    const int k = step_groups(st);
    return k > 1 ? st_step_grouped(st, k) : st_step_device(st);
}

// Groups of engines that engine_batch_step pipelines (0: automatic).
extern "C" int engine_batch_setgroups(struct engine_batch* b, int groups) {
    if (b == nullptr) return engine_err_null;
    if (groups < 0 || groups > 64) return engine_err_range;
    bstate(b)->groups_req = groups;
    return 0;
}

extern "C" int engine_batch_step_host(struct engine_batch* b) {
    if (b == nullptr) return engine_err_null;
    NbState* st = bstate(b);
    for (struct engine* e : st->engines)
        if (e->nr_bonds > 0 || e->nr_angles > 0 || e->nr_dihedrals > 0)   // bonded: device steps only
            return engine_err = engine_err_nyi;
    for (struct engine* e : st->engines) {
        e->time += 1;
        if (space_shuffle(&e->s) < 0) return engine_err = engine_err_space;
    }
    const int rc = st_nonbond(st, true);
    if (rc < 0) return rc;
    for (struct engine* e : st->engines) {
        e->s.epot += e->s.epot_nonbond;
        if (engine_advance(e) < 0) return engine_err;
        if (e->nr_rigids > 0 && engine_rigid_eval(e) < 0) return engine_err = engine_err_rigid;
    }
    return 0;
}

// engine_zero_forces for every engine of the batch (host threads over the cells).
extern "C" int engine_batch_resident_begin(struct engine_batch* b, int margin) {
    if (b == nullptr) return engine_err_null;
    const int rc = st_resident_begin(bstate(b), margin, 16);
    return rc < 0 ? rc : elog_restart(bstate(b));
}

extern "C" int engine_batch_resident_steps(struct engine_batch* b, int nsteps) {
    if (b == nullptr) return engine_err_null;
    return st_resident_steps(bstate(b), nsteps);
}

extern "C" int engine_batch_resident_sync(struct engine_batch* b) {
    if (b == nullptr) return engine_err_null;
    return st_resident_sync(bstate(b));
}

extern "C" int engine_batch_resident_info(struct engine_batch* b, int* capc, int* mcap, long long* steps,
                                          long long* pairs, int* regrows) {
    if (b == nullptr) return engine_err_null;
    return st_resident_info(bstate(b), capc, mcap, steps, pairs, regrows);
}

extern "C" int engine_batch_resident_end(struct engine_batch* b) {
    if (b == nullptr) return engine_err_null;
    NbState* st = bstate(b);
    int rc = st->res_active ? st_resident_sync(st) : 0;
    res_free(st);
    return rc;
}

extern "C" int engine_batch_zero_forces(struct engine_batch* b) {
    if (b == nullptr) return engine_err_null;
    NbState* st = bstate(b);
    for (struct engine* e : st->engines) {
        struct space* s = &e->s;
        s->epot = s->epot_nonbond = s->epot_bond = s->epot_angle = s->epot_dihedral = s->epot_exclusion = 0.0;
    }
    HostPool::get().run(st->ncells, cell_grain(st), [&](int, int cb, int ce) {
        for (int c = cb; c < ce; c++) {
            struct cell* cl = st->flat_cells[c];
            cl->epot = 0.0;
            for (int q = 0; q < cl->count; q++) cl->parts[q].f[0] = cl->parts[q].f[1] = cl->parts[q].f[2] = 0.0f;
        }
    });
    return 0;
}

extern "C" int engine_batch_stats(struct engine_batch* b, struct nb_stats* out) {
    if (b == nullptr || out == nullptr) return engine_err_null;
    *out = bstate(b)->bstats;
    return 0;
}

extern "C" int engine_batch_setstream(struct engine_batch* b, void* stream) {
    if (b == nullptr) return engine_err_null;
    return st_setstream(bstate(b), stream);
}

extern "C" int engine_batch_kernel_times(struct engine_batch* b, float* total_ms, float* sweep_ms) {
    if (b == nullptr) return engine_err_null;
    return st_kernel_times(bstate(b), total_ms, sweep_ms);
}

extern "C" int engine_batch_settune(struct engine_batch* b, int warps, int plain) {
    if (b == nullptr) return engine_err_null;
    return st_settune(bstate(b), warps, plain);
}

extern "C" int engine_batch_graph(struct engine_batch* b, int enable) {
    if (b == nullptr) return engine_err_null;
    NbState* st = bstate(b);
    st->use_graph = enable != 0;
    if (!st->use_graph) drop_graph(st);
    st->prepared_key = -1;
    return 0;
}

extern "C" int engine_batch_autotune(struct engine_batch* b, int reps, int* warps, int* layout, int* stages,
                                     int* occupancy, float* ms) {
    if (b == nullptr) return engine_err_null;
    return st_autotune(bstate(b), reps, warps, layout, stages, occupancy, ms);
}

extern "C" int engine_batch_setlayout(struct engine_batch* b, int layout, int stages, int occupancy) {
    if (b == nullptr) return engine_err_null;
    return st_setlayout(bstate(b), layout, stages, occupancy);
}

extern "C" int engine_batch_ntasks(struct engine_batch* b) {
    if (b == nullptr) return engine_err_null;
    return bstate(b)->ntasks;
}

namespace {
// Independent FMA chains: 2 flops per lane per FMA, no memory traffic in the loop.
__global__ void __launch_bounds__(256) fma_probe(float* out, int iters, float a, float b) {
    float x0 = threadIdx.x * 1e-3f, x1 = x0 + 1.f, x2 = x0 + 2.f, x3 = x0 + 3.f;
    float x4 = x0 + 4.f, x5 = x0 + 5.f, x6 = x0 + 6.f, x7 = x0 + 7.f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
        }
    }
    const float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == 12345.678f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}
}  // namespace

// Measured FP32 FMA throughput of the current device (TFLOP/s), for roofline fractions.
extern "C" int engine_cuda_fp32_peak(int device, float* tflops) {
    if (tflops == nullptr) return engine_err_null;
    CU(cudaSetDevice(device));
    int sms = 0;
    CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int blocks = sms * 8, threads = 256, iters = 4096;
    float* out = nullptr;
    CU(cudaMalloc(&out, sizeof(float) * blocks * threads));
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    fma_probe<<<blocks, threads>>>(out, 64, 0.999f, 1e-4f);
    float best = 0.f;
    for (int rep = 0; rep < 5; ++rep) {
        CU(cudaEventRecord(e0));
        fma_probe<<<blocks, threads>>>(out, iters, 0.999f, 1e-4f);
        CU(cudaEventRecord(e1));
        CU(cudaEventSynchronize(e1));
        float ms = 0.f;
        CU(cudaEventElapsedTime(&ms, e0, e1));
        const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
        const float tf = (float)(flops / (ms * 1e-3) / 1e12);
        if (tf > best) best = tf;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *tflops = best;
    return 0;
}

namespace {
int st_setorder(NbState* st, const int* order, int n) {
    if (n != st->ntasks) return engine_err_range;
    std::vector<char> seen(n, 0);
    for (int k = 0; k < n; k++) {
        if (order[k] < 0 || order[k] >= n || seen[order[k]]) return engine_err_range;
        seen[order[k]] = 1;
    }
    CU(cudaSetDevice(st->device));
    CU(cudaStreamSynchronize(st->stream));
    CU(cudaMemcpy(st->d_order, order, sizeof(int) * n, cudaMemcpyHostToDevice));
    return 0;
}
}  // namespace

// Replaces the task queue order (a permutation of 0..nr_tasks-1).
extern "C" int engine_cuda_setorder(struct engine* e, const int* order, int n) {
    if (e == nullptr || e->cuda == nullptr || order == nullptr) return engine_err_null;
    return st_setorder(state(e), order, n);
}

// The current queue order (task indices in scheduling order).
extern "C" int engine_cuda_getorder(struct engine* e, int* order, int n) {
    if (e == nullptr || e->cuda == nullptr || order == nullptr) return engine_err_null;
    NbState* st = state(e);
    if (n != st->ntasks) return engine_err_range;
    CU(cudaSetDevice(st->device));
    CU(cudaStreamSynchronize(st->stream));
    CU(cudaMemcpy(order, st->d_order, sizeof(int) * n, cudaMemcpyDeviceToHost));
    return 0;
}

// Switches per-task clock64 recording on or off; reads the last launch's records
// (start, end, SM of every task) when the output pointers are given.
extern "C" int engine_cuda_taskclocks(struct engine* e, int enable, long long* clocks, int* sms, int n) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    NbState* st = state(e);
    CU(cudaSetDevice(st->device));
    CU(cudaStreamSynchronize(st->stream));
    if (clocks != nullptr || sms != nullptr) {
        if (n != st->ntasks) return engine_err_range;
        if (clocks) CU(cudaMemcpy(clocks, st->d_task_clock, sizeof(long long) * 2 * n, cudaMemcpyDeviceToHost));
        if (sms) CU(cudaMemcpy(sms, st->d_task_sm, sizeof(int) * n, cudaMemcpyDeviceToHost));
    }
    st->record_clock = enable ? 1 : 0;
    return 0;
}

extern "C" int engine_cuda_ntasks(struct engine* e) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    return state(e)->ntasks;
}

// ---------------------------------------------------------------- allocation-free variant
//
// Some callers cannot allocate device memory at the time they need forces: a host
// program that hands this engine a fixed device-memory budget (every byte pre-reserved by
// its own allocator), a caller inside a region where a cudaMalloc would synchronise the
// device or is forbidden (real-time loops, code running between the engine's set-up and a
// stream capture), or a plugin that must not grow the process's footprint.  For them,
// engine_nonbond_cuda_noalloc runs the same sort + persistent sweep on caller-provided
// device buffers and keeps its only scratch -- the sort key lists, the task-queue head and
// a layout-error word -- in the file-scope array below, sized for at most
// kNoAllocMaxSlots particle slots.  Every GPU that loads this library holds the array
// until the process exits.
//
// The array's name is a host-side stand-in, not a device address; the first call on each
// device (with that device current) looks the address up with cudaGetSymbolAddress.  That
// first call should therefore come before any stream capture.  All calls share the one
// array and it keeps the last call's contents: the queue head and the layout-error word
// are cleared on every call, and calls that overlap on the GPU (other streams, other host
// threads) race on it.
//
// The call touches none of the launch state the engine's own evaluations keep (the
// persistent grid of the last direct launch, the captured graphs): it sizes its own grid
// and only ever raises the sweep kernel's shared-memory limit, so evaluations through
// engine_nonbond_cuda before and after it, with or without graphs, are unaffected.

namespace {
constexpr int kNoAllocMaxSlots = 65536;
constexpr size_t kNoAllocKeyBytes = (size_t)13 * kNoAllocMaxSlots * sizeof(unsigned);
static __device__ __align__(256) unsigned char noalloc_scratch[kNoAllocKeyBytes + 256];

constexpr int kMaxDevices = 64;
unsigned char* noalloc_addr[kMaxDevices] = {nullptr};

// Checks every cell against the layout the bulk copies rely on: a start that is a multiple
// of 4 slots and a 4-rounded block inside [0, nslots).  A bad cell sets the status bit and
// the abort word, and the sort and sweep that follow return without touching memory.
__global__ void noalloc_check_cells(const int* __restrict__ cstart, const int* __restrict__ ccount, int ncells,
                                    int nslots, unsigned long long* __restrict__ acc,
                                    unsigned long long* __restrict__ abort) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    const long long s = cstart[c], n = ccount[c];
    if ((s & 3) != 0 || s < 0 || n < 0 || s + ((n + 3) & ~3LL) > nslots) {
        atomicOr(&acc[kAccStatus], (unsigned long long)kStatusLayout);
        atomicExch(abort, 1ull);
    }
}

template <int NW, bool EX, int TAB>
int noalloc_sweep_nw(const NbState* st, const TunedParams& T, int cap, size_t smem, cudaStream_t s) {
    auto kern = sweep_tuned<NW, EX, TAB, 4, 1, 640, false>;
    cudaFuncAttributes fa;
    CU(cudaFuncGetAttributes(&fa, kern));
    if (fa.maxDynamicSharedSizeBytes < (int)smem)
        CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NW * 32, smem));
    kern<<<st->sm_count * std::max(1, per_sm), NW * 32, smem, s>>>(T, cap);
    CU(cudaGetLastError());
    return 0;
}

template <int NW>
int noalloc_sweep(const NbState* st, const TunedParams& T, int cap, size_t smem, cudaStream_t s) {
    if (st->tab_global)
        return st->has_excl ? noalloc_sweep_nw<NW, true, kTabGlobal>(st, T, cap, smem, s)
                            : noalloc_sweep_nw<NW, false, kTabGlobal>(st, T, cap, smem, s);
    if (st->has_excl)
        return st->one_pot ? noalloc_sweep_nw<NW, true, kTabOne>(st, T, cap, smem, s)
                           : noalloc_sweep_nw<NW, true, kTabShared>(st, T, cap, smem, s);
    return st->one_pot ? noalloc_sweep_nw<NW, false, kTabOne>(st, T, cap, smem, s)
                       : noalloc_sweep_nw<NW, false, kTabShared>(st, T, cap, smem, s);
}

int noalloc_fail(int code, const char* msg, int line) {
    errs_register(code, msg, line, "engine_nonbond_cuda_noalloc", __FILE__);
    return engine_err = code;
}

int nonbond_noalloc(struct engine* e, const void* xq, const int* pid, const int* cstart, const int* ccount,
                    int nslots, int maxcount, unsigned long long* force, unsigned long long* cell_epot,
                    unsigned long long* acc, void* stream) {
    NbState* st = state(e);
    if (nslots < 0 || nslots > kNoAllocMaxSlots)
        return noalloc_fail(engine_err_range, "engine_nonbond_cuda_noalloc: more particle slots than its 65536-slot scratch.",
                            __LINE__);
    if (maxcount < 0 || maxcount > kMaxPartsPerCell)
        return noalloc_fail(engine_err_maxparts, "engine_nonbond_cuda_noalloc: cell larger than 1024 particles.", __LINE__);
    if ((((uintptr_t)xq | (uintptr_t)pid) & 15) != 0 || (((uintptr_t)force | (uintptr_t)cell_epot | (uintptr_t)acc) & 7) != 0 ||
        (((uintptr_t)cstart | (uintptr_t)ccount) & 3) != 0)
        return noalloc_fail(engine_err_range,
                            "engine_nonbond_cuda_noalloc: xq and pid must be 16-byte aligned, force, cell_epot and acc 8-byte "
                            "aligned, cstart and ccount 4-byte aligned.",
                            __LINE__);
    if (st->device < 0 || st->device >= kMaxDevices)
        return noalloc_fail(engine_err_range, "engine_nonbond_cuda_noalloc: device index out of range.", __LINE__);

    // Launch shape, decided before any work is queued: 4 worker warps, 2 when the warps'
    // staging slices of the largest cell would not leave room for a second block.
    const int cap4 = (maxcount + 3) & ~3;
    const int cap = cap4 + 8;
    const int tc = st->tab_global ? 0 : st->ncoef, tp = st->tab_global ? 0 : st->npots;
    int nw = 4;
    size_t smem = warps_smem_bytes(cap, nw, tc, tp, st->max_type, 1);
    if (smem > 200 * 1024) {
        nw = 2;
        smem = warps_smem_bytes(cap, nw, tc, tp, st->max_type, 1);
    }
    if (smem > 220 * 1024)
        return noalloc_fail(engine_err_maxparts, "Cell too large for the sweep kernel's shared memory.", __LINE__);

    CU(cudaSetDevice(st->device));
    if (noalloc_addr[st->device] == nullptr) {
        void* p = nullptr;
        CU(cudaGetSymbolAddress(&p, noalloc_scratch));
        noalloc_addr[st->device] = static_cast<unsigned char*>(p);
    }
    unsigned* keys = reinterpret_cast<unsigned*>(noalloc_addr[st->device]);
    int* counter = reinterpret_cast<int*>(noalloc_addr[st->device] + kNoAllocKeyBytes);
    unsigned long long* abort = reinterpret_cast<unsigned long long*>(noalloc_addr[st->device] + kNoAllocKeyBytes + 8);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : st->stream;

    CU(cudaMemsetAsync(force, 0, sizeof(unsigned long long) * 3 * (size_t)nslots, s));
    CU(cudaMemsetAsync(cell_epot, 0, sizeof(unsigned long long) * st->ncells, s));
    CU(cudaMemsetAsync(acc, 0, sizeof(unsigned long long) * kAccCount, s));
    CU(cudaMemsetAsync(counter, 0, 16, s));                  // queue head and abort word
    if (cap4 == 0 || st->ncells == 0) return 0;
    noalloc_check_cells<<<(st->ncells + 255) / 256, 256, 0, s>>>(cstart, ccount, st->ncells, nslots, acc, abort);
    CU(cudaGetLastError());
    const int cpc = sort_cells_per_block(nslots, st->ncells);
    const int rcs = launch_sort(static_cast<const float4*>(xq), cstart, ccount, st->d_cmask, keys, st->d_cscale,
                                st->ncells, cpc, cap4, acc, abort, false, s);
    if (rcs < 0) return rcs;

    TunedParams T;
    Params& P = T.p;
    P.xq = static_cast<const float4*>(xq);
    P.pid = pid;
    P.keys = keys;
    P.cstart = cstart;
    P.ccount = ccount;
    P.force = force;
    P.acc = acc;
    P.cell_epot = cell_epot;
    P.cell_vir = nullptr;
    P.tasks = st->d_tasks;
    P.tshift = st->d_tshift;
    P.ntasks = st->ntasks;
    P.coef = st->d_coef;
    P.potinfo = st->d_potinfo;
    P.potn = st->d_potn;
    P.potidx = st->d_potidx;
    P.max_type = st->max_type;
    P.npots = st->npots;
    P.ncoef = st->ncoef;
    P.emask = st->d_emask;
    P.exoff = st->d_exoff;
    P.exlist = st->d_exlist;
    const float cutf = (float)e->s.cutoff;
    P.cutoff2 = cutf * cutf;
    P.cutoff2s = (float)e->s.cutoff2;
    P.unsorted = (e->flags & engine_flag_unsorted) ? 1 : 0;
    P.abort = abort;
    P.qid = st->d_qid;
    P.ep_pot = st->ep_pot;
    P.tab_global = st->tab_global;
    P.tiny = tiny_tasks_of(st);
    T.order = st->d_order;
    T.qcount = nullptr;
    T.counter = counter;
    T.task_clock = nullptr;
    T.task_sm = nullptr;
    return nw == 2 ? noalloc_sweep<2>(st, T, cap, smem, s) : noalloc_sweep<4>(st, T, cap, smem, s);
}
}  // namespace

extern "C" int engine_nonbond_cuda_noalloc(struct engine* e, const void* xq, const int* pid, const int* cstart,
                                           const int* ccount, int nslots, int maxcount,
                                           unsigned long long* force, unsigned long long* cell_epot,
                                           unsigned long long* acc, void* stream) {
    if (e == nullptr || e->cuda == nullptr || xq == nullptr || pid == nullptr || cstart == nullptr ||
        ccount == nullptr || force == nullptr || cell_epot == nullptr || acc == nullptr)
        return noalloc_fail(engine_err_null, "engine_nonbond_cuda_noalloc: NULL argument.", __LINE__);
    // The caller's current device is restored on return.
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    const int rc = nonbond_noalloc(e, xq, pid, cstart, ccount, nslots, maxcount, force, cell_epot, acc, stream);
    if (prev >= 0) cudaSetDevice(prev);
    return rc;
}

// ---------------------------------------------------------------- learned scheduler
namespace {

// Per-cell count of type-0 particles (the type mix feature).
__global__ void cell_type0(const float4* __restrict__ xq, const int* __restrict__ cstart,
                           const int* __restrict__ ccount, int ncells, int* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    int n0 = 0;
    for (int k = 0; k < ccount[c]; k++) n0 += __float_as_int(xq[cstart[c] + k].w) == 0;
    out[c] = n0;
}

// Features of every task (NB_MLP_IN floats): counts, reach fraction, pair volume, type mix,
// neighbour class one-hot (face, edge, corner, self).
__global__ void task_features(const TaskRec* __restrict__ tasks, int ntasks, const int* __restrict__ ccount,
                              const int* __restrict__ cstart, const unsigned* __restrict__ keys,
                              const int* __restrict__ ctype0, float inv_scale,
                              float* __restrict__ X) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntasks) return;
    const TaskRec r = tasks[t];
    const int ni = ccount[r.ci], nj = ccount[r.cj];
    float reach = 1.f;
    int cls = 3;
    if (r.sid >= 0) {
        const int idx = 26 - r.sid;
        cls = (idx / 9 != 1) + ((idx / 3) % 3 != 1) + (idx % 3 != 1) - 1;
        if (ni > 0 && nj > 0) {
            const int padi = (ni + 3) & ~3, padj = (nj + 3) & ~3;
            const unsigned* ki = keys + 13 * (size_t)cstart[r.ci] + (size_t)r.sid * padi;
            const unsigned* kj = keys + 13 * (size_t)cstart[r.cj] + (size_t)r.sid * padj;
            const int thr = (int)(kj[nj - 1] & 0xffffu) + task_dnshift(r) - task_dmax(r);   // i needs dist >= thr
            int lo = 0, hi = ni;                                                   // descending list
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if ((int)(ki[mid] & 0xffffu) >= thr) lo = mid + 1; else hi = mid;
            }
            reach = (float)lo / (float)ni;
        } else {
            reach = 0.f;
        }
    }
    float* x = X + (size_t)t * NB_MLP_IN;
    x[0] = ni * inv_scale;
    x[1] = nj * inv_scale;
    x[2] = reach;
    x[3] = (float)ni * (float)nj * reach * inv_scale * inv_scale;
    x[4] = ni > 0 ? (float)ctype0[r.ci] / ni : 0.f;
    x[5] = nj > 0 ? (float)ctype0[r.cj] / nj : 0.f;
    for (int k = 0; k < 4; k++) x[6 + k] = (k == cls) ? 1.f : 0.f;
}

// Adds this launch's task durations (clock64 cycles) into the running sums.
__global__ void accumulate_durations(const long long* __restrict__ clk, int ntasks, double* __restrict__ dur,
                                     int* __restrict__ nrec) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntasks) return;
    const long long a = clk[2 * t], b = clk[2 * t + 1];
    if (b > a && a > 0) {
        dur[t] += (double)(b - a);
        nrec[t] += 1;
    }
}

struct SchedState {
    float* d_feat = nullptr;
    double* d_dur = nullptr;
    int* d_nrec = nullptr;
    int* d_ctype0 = nullptr;
    float* d_target = nullptr;
    float* d_pred = nullptr;
    int* d_idx = nullptr;
    float *d_wm = nullptr, *d_m = nullptr, *d_v = nullptr, *d_grad = nullptr, *d_loss = nullptr;
    void* d_wb = nullptr;
    int step = 0;
    bool trained = false;
    std::vector<int> heuristic;   // count-product order
};

SchedState* sched(struct engine* e, NbState* st);

}  // namespace

#include <random>

extern "C" int nb_mlp_predict(const float* X, int n, const void* w_bf16, float* out, void* stream);
extern "C" int nb_mlp_grad(const float* X, const float* target, const int* idx, int n, const void* w_bf16,
                           float* grad, float* loss, void* stream);
extern "C" int nb_mlp_adam(float* w_master, void* w_bf16, const float* grad, float* m, float* v, float lr,
                           float beta1, float beta2, float eps, int step, void* stream);
extern "C" int nb_mlp_round(const float* w_master, void* w_bf16, void* stream);

namespace {

void sched_free(void* p) {
    SchedState* ss = static_cast<SchedState*>(p);
    if (ss == nullptr) return;
    void* bufs[] = {ss->d_feat, ss->d_dur, ss->d_nrec, ss->d_ctype0, ss->d_target, ss->d_pred, ss->d_idx,
                    ss->d_wm, ss->d_m, ss->d_v, ss->d_grad, ss->d_loss, ss->d_wb};
    for (void* b : bufs) cudaFree(b);
    delete ss;
}

SchedState* sched(struct engine* e, NbState* st) {
    (void)e;
    if (st->sched) return static_cast<SchedState*>(st->sched);
    SchedState* ss = new SchedState();
    st->sched = ss;
    const int n = st->ntasks > 0 ? st->ntasks : 1;
    bool bad = dev_alloc(&ss->d_feat, (size_t)n * NB_MLP_IN) || dev_alloc(&ss->d_dur, n) ||
               dev_alloc(&ss->d_nrec, n) || dev_alloc(&ss->d_ctype0, st->ncells) || dev_alloc(&ss->d_target, n) ||
               dev_alloc(&ss->d_pred, n) || dev_alloc(&ss->d_idx, n) || dev_alloc(&ss->d_wm, NB_MLP_NPARAM) ||
               dev_alloc(&ss->d_m, NB_MLP_NPARAM) || dev_alloc(&ss->d_v, NB_MLP_NPARAM) ||
               dev_alloc(&ss->d_grad, NB_MLP_NPARAM) || dev_alloc(&ss->d_loss, 1);
    if (!bad) bad = cudaMalloc(&ss->d_wb, sizeof(uint16_t) * NB_MLP_NPARAM) != cudaSuccess;
    if (bad) return nullptr;
    cudaMemset(ss->d_dur, 0, sizeof(double) * n);
    cudaMemset(ss->d_nrec, 0, sizeof(int) * n);
    return ss;
}

}  // namespace

// Runs nsteps device-resident evaluations with per-task clock64 records and adds each
// task's duration into a running sum (the training targets).
extern "C" int engine_sched_record(struct engine* e, int nsteps) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    NbState* st = state(e);
    CU(cudaSetDevice(st->device));
    SchedState* ss = sched(e, st);
    if (ss == nullptr) return engine_err_cuda;
    if (!st->resident_valid && !st->res_active) {
        int rc = engine_cuda_load_parts(e);
        if (rc < 0) return rc;
    }
    const int prev = st->record_clock;
    st->record_clock = 1;
    for (int k = 0; k < nsteps; k++) {
        CU(cudaMemsetAsync(st->d_task_clock, 0, sizeof(long long) * 2 * st->ntasks, st->stream));
        // device-resident particles: one MD step each (the trajectory advances); else one
        // force evaluation of the uploaded particles
        int rc = st->res_active ? st_resident_steps(st, 1) : launch_kernels(st);
        if (rc < 0) {
            st->record_clock = prev;
            return rc;
        }
        accumulate_durations<<<(st->ntasks + 255) / 256, 256, 0, st->stream>>>(st->d_task_clock, st->ntasks,
                                                                             ss->d_dur, ss->d_nrec);
        CU(cudaGetLastError());
    }
    st->record_clock = prev;
    CU(cudaStreamSynchronize(st->stream));
    return 0;
}

// Features of the current configuration (needs the sort keys of the last launch).
extern "C" int engine_sched_features(struct engine* e, float* features_out, int n) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    NbState* st = state(e);
    CU(cudaSetDevice(st->device));
    SchedState* ss = sched(e, st);
    if (ss == nullptr) return engine_err_cuda;
    // the particles and sort keys of the last evaluation: the resident cells' current side
    // during device-resident steps, else the uploaded particles
    const bool res = st->res_active;
    const float4* xq = res ? st->r_xq[st->rside] : st->d_xq;
    const int* cstart = res ? st->r_cstart : st->d_cstart;
    const int* ccount = res ? st->r_cnt[st->rside] : st->d_ccount;
    const unsigned* keys = res ? st->r_keys : st->d_keys;
    cell_type0<<<(st->ncells + 255) / 256, 256, 0, st->stream>>>(xq, cstart, ccount, st->ncells, ss->d_ctype0);
    task_features<<<(st->ntasks + 255) / 256, 256, 0, st->stream>>>(st->d_tasks, st->ntasks, ccount, cstart, keys,
                                                                    ss->d_ctype0, 1.0f / 32.0f, ss->d_feat);
    CU(cudaGetLastError());
    if (features_out != nullptr) {
        if (n != st->ntasks) return engine_err_range;
        CU(cudaMemcpyAsync(features_out, ss->d_feat, sizeof(float) * NB_MLP_IN * (size_t)n, cudaMemcpyDeviceToHost,
                           st->stream));
    }
    CU(cudaStreamSynchronize(st->stream));
    return 0;
}

// Mean recorded duration per task normalised by the mean over recorded tasks (0 for tasks
// that never ran, e.g. with an empty cell); uploads them as training targets.
extern "C" int engine_sched_targets(struct engine* e, float* targets_out, int n) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    NbState* st = state(e);
    CU(cudaSetDevice(st->device));
    SchedState* ss = sched(e, st);
    if (ss == nullptr) return engine_err_cuda;
    std::vector<double> dur(st->ntasks);
    std::vector<int> nrec(st->ntasks);
    CU(cudaMemcpy(dur.data(), ss->d_dur, sizeof(double) * st->ntasks, cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(nrec.data(), ss->d_nrec, sizeof(int) * st->ntasks, cudaMemcpyDeviceToHost));
    double sum = 0.0;
    int cnt = 0;
    for (int t = 0; t < st->ntasks; t++)
        if (nrec[t] > 0) { sum += dur[t] / nrec[t]; cnt++; }
    const double mean = cnt ? sum / cnt : 1.0;
    std::vector<float> tg(st->ntasks);
    for (int t = 0; t < st->ntasks; t++) tg[t] = nrec[t] > 0 ? (float)(dur[t] / nrec[t] / mean) : 0.f;
    CU(cudaMemcpy(ss->d_target, tg.data(), sizeof(float) * st->ntasks, cudaMemcpyHostToDevice));
    if (targets_out != nullptr) {
        if (n != st->ntasks) return engine_err_range;
        std::copy(tg.begin(), tg.end(), targets_out);
    }
    return 0;
}

// Adam on mini-batches of the recorded tasks (at most 2^18 samples per epoch), weights
// initialised on the first call (He-normal, seeded).
extern "C" int engine_sched_train(struct engine* e, int epochs, int batch, float lr, unsigned seed, float* loss_out) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    NbState* st = state(e);
    CU(cudaSetDevice(st->device));
    SchedState* ss = sched(e, st);
    if (ss == nullptr) return engine_err_cuda;
    std::mt19937 rng(seed);
    if (!ss->trained && ss->step == 0) {
        std::vector<float> w(NB_MLP_NPARAM, 0.f);
        auto fill = [&](int off, int nout, int nin) {
            std::normal_distribution<float> nd(0.f, std::sqrt(2.f / nin));
            for (int k = 0; k < nout * nin; k++) w[off + k] = nd(rng);
        };
        const int H = NB_MLP_HIDDEN, I = NB_MLP_IN;
        fill(0, H, I);
        fill(H * I + H, H, H);
        fill(H * I + H + H * H + H, 1, H);
        w[NB_MLP_NPARAM - 1] = 1.0f;                   // targets are normalised to mean 1
        CU(cudaMemcpy(ss->d_wm, w.data(), sizeof(float) * NB_MLP_NPARAM, cudaMemcpyHostToDevice));
        CU(cudaMemset(ss->d_m, 0, sizeof(float) * NB_MLP_NPARAM));
        CU(cudaMemset(ss->d_v, 0, sizeof(float) * NB_MLP_NPARAM));
        if (nb_mlp_round(ss->d_wm, ss->d_wb, st->stream) < 0) return engine_err_cuda;
    }
    const int n = st->ntasks;
    std::vector<int> perm(n);
    for (int k = 0; k < n; k++) perm[k] = k;
    const int per_epoch = std::min(n, 1 << 18);
    if (batch <= 0) batch = 1024;
    for (int ep = 0; ep < epochs; ep++) {
        std::shuffle(perm.begin(), perm.end(), rng);
        CU(cudaMemcpyAsync(ss->d_idx, perm.data(), sizeof(int) * per_epoch, cudaMemcpyHostToDevice, st->stream));
        CU(cudaStreamSynchronize(st->stream));
        for (int b0 = 0; b0 < per_epoch; b0 += batch) {
            const int nb = std::min(batch, per_epoch - b0);
            if (nb_mlp_grad(ss->d_feat, ss->d_target, ss->d_idx + b0, nb, ss->d_wb, ss->d_grad, ss->d_loss,
                            st->stream) < 0)
                return engine_err_cuda;
            if (nb_mlp_adam(ss->d_wm, ss->d_wb, ss->d_grad, ss->d_m, ss->d_v, lr, 0.9f, 0.999f, 1e-8f, ++ss->step,
                            st->stream) < 0)
                return engine_err_cuda;
        }
    }
    ss->trained = true;
    if (loss_out != nullptr) {
        // mean squared error over every task
        if (nb_mlp_grad(ss->d_feat, ss->d_target, nullptr, n, ss->d_wb, ss->d_grad, ss->d_loss, st->stream) < 0)
            return engine_err_cuda;
        CU(cudaMemcpyAsync(loss_out, ss->d_loss, sizeof(float), cudaMemcpyDeviceToHost, st->stream));
    }
    CU(cudaStreamSynchronize(st->stream));
    return 0;
}

extern "C" int engine_sched_predict(struct engine* e, float* pred_out, int n) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    NbState* st = state(e);
    CU(cudaSetDevice(st->device));
    SchedState* ss = sched(e, st);
    if (ss == nullptr || !ss->trained) return engine_err_range;
    if (nb_mlp_predict(ss->d_feat, st->ntasks, ss->d_wb, ss->d_pred, st->stream) < 0) return engine_err_cuda;
    if (pred_out != nullptr) {
        if (n != st->ntasks) return engine_err_range;
        CU(cudaMemcpyAsync(pred_out, ss->d_pred, sizeof(float) * n, cudaMemcpyDeviceToHost, st->stream));
    }
    CU(cudaStreamSynchronize(st->stream));
    return 0;
}

namespace {

// Task costs of the current configuration: predicted by the network (source 1) or the
// reference's count-product weights (source 0, src/engine.c:574-576, 643-699).
int task_costs(struct engine* e, NbState* st, int source, std::vector<float>& cost) {
    cost.assign(st->ntasks, 0.f);
    if (source == 1) return engine_sched_predict(e, cost.data(), st->ntasks);
    std::vector<int> cnt(st->ncells);
    if (st->res_active) {
        CU(cudaStreamSynchronize(st->stream));
        CU(cudaMemcpy(cnt.data(), st->r_cnt[st->rside], sizeof(int) * st->ncells, cudaMemcpyDeviceToHost));
    } else {
        for (size_t k = 0; k < st->engines.size(); k++)
            for (int c = 0; c < st->engines[k]->s.nr_cells; c++)
                cnt[st->cell_off[k] + c] = st->engines[k]->s.cells[c].count;
    }
    std::vector<TaskRec> tasks(st->ntasks);
    CU(cudaMemcpy(tasks.data(), st->d_tasks, sizeof(TaskRec) * st->ntasks, cudaMemcpyDeviceToHost));
    for (int t = 0; t < st->ntasks; t++) cost[t] = (float)task_weight(tasks[t].sid, cnt[tasks[t].ci], cnt[tasks[t].cj]);
    return 0;
}

}  // namespace

// Orders the queue from task costs with locality: the tasks, in the cell-major order they
// were generated in, are cut into tiles of `tile` consecutive tasks (0: about an eighth of
// the tasks per worker warp of the persistent sweep, so that every warp still takes several
// tiles); each tile's cost is the sum of its tasks' costs, and the tiles go in decreasing
// cost class (a factor of 2^(1/4) per class) and, within a class, in cell-major order, each
// tile's tasks by decreasing cost.  Longest-first at tile granularity, so that the queue
// ends with cheap work, while neighbouring cells are swept close together in time and their
// particles are read from L2 rather than DRAM.  tile = 1 is plain longest-first.
namespace {
int st_sched_order(NbState* st, struct engine* e, int source, int tile) {
    if ((source != 0 && source != 1) || tile < 0 || (source == 1 && e == nullptr)) return engine_err_range;
    CU(cudaSetDevice(st->device));
    std::vector<float> cost;
    int rc = task_costs(e, st, source, cost);
    if (rc < 0) return rc;
    const int n = st->ntasks;
    if (tile == 0) tile = auto_tile(n, st->sm_count, st->occupancy);
    const std::vector<int> order = tiled_order(std::vector<double>(cost.begin(), cost.end()), n, tile);
    return st_setorder(st, order.data(), n);
}
}  // namespace

extern "C" int engine_sched_order(struct engine* e, int source, int tile) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    return st_sched_order(state(e), e, source, tile);
}

// The same locality-tiled order for a batch, from the count-product costs (the tasks of
// each engine are consecutive, cell-major, so tiles stay inside one engine's box).
extern "C" int engine_batch_sched_order(struct engine_batch* b, int tile) {
    if (b == nullptr) return engine_err_null;
    return st_sched_order(bstate(b), nullptr, 0, tile);
}

// Orders the queue by decreasing predicted cost (use_mlp) or restores the count-product
// heuristic order.
extern "C" int engine_sched_apply(struct engine* e, int use_mlp) {
    if (e == nullptr || e->cuda == nullptr) return engine_err_null;
    NbState* st = state(e);
    CU(cudaSetDevice(st->device));
    if (!use_mlp) return engine_cuda_setorder(e, st->heur_order.data(), st->ntasks);
    std::vector<float> pred(st->ntasks);
    int rc = engine_sched_predict(e, pred.data(), st->ntasks);
    if (rc < 0) return rc;
    std::vector<int> order(st->ntasks);
    for (int t = 0; t < st->ntasks; t++) order[t] = t;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return pred[a] > pred[b]; });
    return engine_cuda_setorder(e, order.data(), st->ntasks);
}
