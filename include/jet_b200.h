/*
 * jet_b200.h -- C ABI of the B200 Jet multilevel k-way graph partitioner.
 *
 * Plain pointers and sizes only.  Every entry point returns a status code
 * (JET_OK on success).  Graph arrays describe a symmetric CSR without
 * self-loops with both edge directions stored, as the reference's
 * KokkosSparse::CrsMatrix input does (header/jet_defs.h:64-92):
 *   row_map[n+1]  edge offsets       entries[nnz]  neighbour ids
 *   values[nnz]   edge weights       vweights[n]   vertex weights
 * Three integer tiers mirror header/jet_defs.h:47-92:
 *   _i32      int32 ordinals, int32 offsets, int32 weights   (jet.h "std")
 *   _big      int32 ordinals, int64 offsets, int64 weights
 *   _biggest  int64 ordinals, int64 offsets, int64 weights
 * Part ids are int32.  `mem` says where the graph and output arrays live:
 * JET_MEM_HOST (the library copies in and out) or JET_MEM_DEVICE (pointers
 * into the current CUDA device's memory).  `stream` is a cudaStream_t (NULL =
 * the library's own stream); calls return after the result is written.
 */
#ifndef JET_B200_H
#define JET_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    JET_OK = 0,
    JET_ERR_INVALID = 1,   /* bad argument or malformed graph */
    JET_ERR_CUDA = 2,      /* CUDA runtime error */
    JET_ERR_METIS = 3,     /* Metis failed on the coarsest graph (the reference exits) */
    JET_ERR_OOM = 4,       /* device allocation failed */
    JET_ERR_OVERFLOW = 5,  /* a hash table ran out of room */
    JET_ERR_TIMEOUT = 6,   /* a bounded device loop gave up */
    JET_ERR_NOT_BUILT = 7  /* no CUDA device / library not usable */
};

enum { JET_MEM_HOST = 0, JET_MEM_DEVICE = 1 };

/* config_t of header/jet_config.h:43-52, field for field. */
typedef struct jet_config_c {
    int32_t coarsening_alg;   /* 0 = 2-hop matching, 1 = HEC, 2 = pure matching */
    int32_t num_iter;         /* used by drivers only (attempt count) */
    double max_imb_ratio;
    int32_t num_parts;
    double refine_tolerance;  /* default 0.999 */
    int32_t dump_coarse;      /* write coarse_graphs.out / coarse_part.out (src/binary_dump.hpp) */
    int32_t verbose;
    int32_t ultra_settings;
} jet_config_c;

/* experiment_data<...>::CoarseLevel, header/experiment_data.hpp:102-123. */
typedef struct jet_level_stats_c {
    int64_t edge_cut;
    double imb;
    uint64_t num_edges;
    uint64_t num_vertices;
    double total_ref_time;
    double iterations_time;
    int32_t total_iterations;
    int32_t lp_iterations;
} jet_level_stats_c;

#define JET_MAX_LEVELS 256
#define JET_NUM_MEASUREMENTS 20

/* experiment_data<...>, header/experiment_data.hpp:76-175.  measurements[]
 * follows the Measurement enum order (coarsen-map ... total), in seconds. */
typedef struct jet_stats_c {
    double measurements[JET_NUM_MEASUREMENTS];
    int32_t num_levels;
    jet_level_stats_c levels[JET_MAX_LEVELS]; /* coarsest first, as refined */
    int64_t edge_cut;        /* final cut, each cut edge once */
    int64_t max_part_cut;    /* filled when verbose */
    int64_t objective;       /* communication volume, filled when verbose */
    double imb_ratio;        /* largest part / optimal size */
    int64_t largest_part;
    int64_t smallest_part;
    int64_t coarsest_vertices;
    int64_t refine_iterations;
} jet_stats_c;

/* ---------------------------------------------------------------- partition
 * Replaces jet_partitioner::partition / partition_big / partition_biggest
 * (header/jet.h:46-51, :67-72, :88-93; bodies src/jet.cpp:47-54,
 * src/jet_big.cpp:47-54, src/jet_biggest.cpp:47-54): coarsen, Metis on the
 * coarsest graph, uncoarsen with Jet refinement.  part_out[n] receives the
 * partition, *edge_cut the cut (each edge once).  `seed` drives the
 * coarsening RNG (the reference seeds from the clock). stats may be NULL. */
int jet_partition_i32(const jet_config_c* config, int32_t n, const int32_t* row_map, const int32_t* entries,
                      const int32_t* values, const int32_t* vweights, int uniform_ew, int mem, uint64_t seed,
                      void* stream, int32_t* part_out, int32_t* edge_cut, jet_stats_c* stats);
int jet_partition_big(const jet_config_c* config, int32_t n, const int64_t* row_map, const int32_t* entries,
                      const int64_t* values, const int64_t* vweights, int uniform_ew, int mem, uint64_t seed,
                      void* stream, int32_t* part_out, int64_t* edge_cut, jet_stats_c* stats);
int jet_partition_biggest(const jet_config_c* config, int64_t n, const int64_t* row_map, const int64_t* entries,
                          const int64_t* values, const int64_t* vweights, int uniform_ew, int mem, uint64_t seed,
                          void* stream, int32_t* part_out, int64_t* edge_cut, jet_stats_c* stats);

/* ---------------------------------------------------------------- hierarchy dump and import
 * With config.dump_coarse set, a partition call writes, as the reference
 * does (src/uncoarsen.hpp:93-111, src/binary_dump.hpp:61-97), the files
 * "coarse_graphs.out" (the levels from the finest down to the first level
 * whose partition is balanced before refinement, in the reference's binary
 * layout with this tier's types) and "coarse_part.out" (that level's
 * partition) in the working directory.
 * jet_refine_hierarchy replaces app/import_coarse.cpp:49-132: it reads such
 * files (NULL paths = those names), refines from their coarsest level down
 * and writes the finest partition to part_out (host memory, part_capacity
 * entries at least; *n_out receives the finest vertex count).  Imported
 * levels are treated as non-uniform, as in the reference. */
int jet_refine_hierarchy(int tier, const jet_config_c* config, const char* graphs_path, const char* part_path, int32_t* part_out,
                         int64_t part_capacity, int64_t* n_out, int64_t* edge_cut, jet_stats_c* stats, void* stream);

/* ---------------------------------------------------------------- batched
 * Many graphs of one tier in one call (no counterpart in the reference,
 * which partitions one graph per call).  Each graph is an independent
 * partition with the same result as the single-graph entry point given the
 * same arguments; `workers` host threads (0 = 8) each drive their own CUDA
 * stream on the current device and pull the next graph (largest nnz first),
 * so kernels of different graphs overlap on the GPU and the host-side Metis
 * calls overlap GPU work (they run in helper processes, because Metis keeps
 * global state).  Workers use the one-CTA level loop and the host loop only.
 * Set CUDA_DEVICE_MAX_CONNECTIONS=32 in the environment before the process
 * creates its CUDA context so that the workers' streams get separate
 * hardware queues.  Array
 * element types follow the tier as in jet_partition_*; `mem` applies to all
 * graphs.  Returns JET_OK when every graph succeeded, else the first failing
 * graph's code (each graph's own code is in its `status`). */
typedef struct jet_graph_desc {
    int64_t n;
    const void* row_map;
    const void* entries;
    const void* values;
    const void* vweights;
    int32_t uniform_ew;
    jet_config_c config;
    uint64_t seed;
    int32_t* part_out;     /* n entries (memory kind as `mem`) */
    int64_t edge_cut;      /* out: the cut, each edge once */
    int32_t status;        /* out: JET_OK or an error code */
    double latency_ms;     /* out: from submission (batch start) to completion */
    char error[112];       /* out: message when status != JET_OK */
} jet_graph_desc;

int jet_partition_batch(int tier, int64_t count, jet_graph_desc* graphs, int mem, int workers);

/* ---------------------------------------------------------------- serving
 * A request loop over the batched executor: requests are queued as they
 * arrive and admitted (oldest first) while a worker is free and the sum of
 * the admitted requests' estimated device footprints stays within
 * `mem_budget_bytes`; admitted requests run concurrently on their own
 * streams.  A request whose estimate alone exceeds the budget is refused
 * with JET_ERR_OOM.  The caller keeps a request's arrays alive until its
 * ticket is waited for.  Results equal those of jet_partition_* for the same
 * arguments, alone or in any mix.  (No counterpart in the reference.) */
typedef struct jet_server jet_server;
typedef struct jet_server_stats {
    int64_t submitted, completed, failed, refused;
    int64_t peak_footprint_bytes;   /* largest admitted sum seen */
    int32_t peak_concurrent;        /* most requests in flight at once */
} jet_server_stats;

jet_server* jet_server_create(int tier, int mem, int workers, int64_t mem_budget_bytes);
/* Queues a copy of *req; returns a ticket >= 0, or -(error code). */
int64_t jet_server_submit(jet_server* srv, const jet_graph_desc* req);
/* Waits up to timeout_ms (< 0: forever) for a ticket.  JET_OK once the
 * request has finished: *out holds it with its outputs and its own result
 * code in out->status, and the ticket is released.  JET_ERR_TIMEOUT when it
 * is not done yet (wait again); JET_ERR_INVALID for an unknown ticket. */
int jet_server_wait(jet_server* srv, int64_t ticket, jet_graph_desc* out, double timeout_ms);
/* Estimated device bytes a request holds while it runs (the admission unit). */
int64_t jet_server_footprint(int tier, int64_t n, int64_t nnz, int32_t num_parts);
int jet_server_stats_get(jet_server* srv, jet_server_stats* out);
/* Finishes every queued request, then frees the server. */
int jet_server_destroy(jet_server* srv);

/* ---------------------------------------------------------------- components
 * Tier-generic entry points over device pointers (tier 0 = i32, 1 = big,
 * 2 = biggest; pointer element types follow the tier).  They expose the hot
 * path's stages one at a time. */

/* One coarsening map (src/contract.hpp:448-492): alg 0 = 2-hop matching
 * (src/heuristics.hpp:427-671 with match_choice 1), 1 = HEC
 * (src/heuristics.hpp:171-262), 2 = pure matching.  map_out[n] receives the
 * fine->coarse map, hn_out[n] (nullable) the initial heavy-neighbour
 * proposals, *nc the coarse vertex count. */
int jet_coarsen_map(int tier, int alg, int level, uint64_t seed, int64_t n, int64_t nnz, const void* row_map,
                    const void* entries, const void* values, const void* vweights, int uniform, void* map_out,
                    void* hn_out, int64_t* nc, void* stream);

/* Contraction under a given map (src/contract.hpp:347-446): crow[nc+1],
 * cadj[>= nnz], cval[>= nnz], cvw[nc]; *cnnz receives the coarse nnz.  Each
 * coarse row lists its neighbours in increasing id (the reference leaves the
 * order to its hash slots, src/contract.hpp:320-327). */
int jet_contract(int tier, int64_t n, int64_t nnz, const void* row_map, const void* entries, const void* values,
                 const void* vweights, const void* map, int64_t nc, void* crow, void* cadj, void* cval, void* cvw,
                 int64_t* cnnz, void* stream);

/* Connectivity tables for a partition (init_conn_data,
 * src/jet_refiner.hpp:958-1048): off[n+1], ent[>= nnz] (part or -1/-2),
 * val[>= nnz], size[n]. */
int jet_conn_build(int tier, int64_t n, int64_t nnz, const void* row_map, const void* entries, const void* values,
                   const int32_t* part, int32_t k, void* off, int32_t* ent, void* val, int32_t* size, void* stream);

/* `iters` refinement iterations at one level from part[] (in/out) with the
 * iteration body of jet_refine (src/jet_refiner.hpp:1106-1120) and no
 * best-state bookkeeping.  sizes[k], *cut (both directions), the tables as
 * jet_conn_build, dest_cache[n], and per iteration moves[i] and kinds[i]
 * (0 LP, 1 weak, 2 strong).  Table outputs may be NULL. */
int jet_refine_iters(int tier, int64_t n, int64_t nnz, const void* row_map, const void* entries, const void* values,
                     const void* vweights, int32_t* part, int32_t k, double imb, double filter_ratio, int32_t iters,
                     void* sizes, int64_t* cut, void* off, int32_t* ent, void* val, int32_t* size, int32_t* dest_cache,
                     int64_t* moves, int32_t* kinds, void* stream);

/* One full jet_refine at a single level (src/jet_refiner.hpp:1050-1142):
 * part[] in/out, *cut (both directions), *iters. */
int jet_refine_level(int tier, int64_t n, int64_t nnz, const void* row_map, const void* entries, const void* values,
                     const void* vweights, int32_t* part, int32_t k, double imb, double tol, int uniform_ew,
                     int64_t* cut, int32_t* iters, void* stream);

/* Partition quality as pstat reports it (app/part_eval.cpp:73-110):
 * out[6] = {cut (each edge once), max part cut, comm size, largest part,
 * smallest part, total vertex weight}. */
int jet_pstat(int tier, int64_t n, int64_t nnz, const void* row_map, const void* entries, const void* values,
              const void* vweights, const int32_t* part, int32_t k, int64_t* out, void* stream);

/* Projection to the finer level (src/uncoarsen.hpp:82-86): fine[i] = coarse[map[i]]. */
int jet_project(int tier, int64_t n_fine, const void* map, const int32_t* coarse, int32_t* fine, void* stream);

/* Same results as jet_pstat, for callers that must not trigger any device
 * allocation: services that reserve the GPU's memory up front for their own
 * pool (a caching allocator holding the whole device, a real-time loop that
 * must never enter the driver's allocator) and forbid the library from
 * allocating later.  No counterpart in the reference.
 * Scratch is a fixed array of about 256 KiB in the library's device module,
 * held by every GPU that loads it until the process exits.  Under CUDA's lazy
 * module loading (the default) the module -- and the array's memory -- is
 * loaded by the first call on each device, which also looks up the array's
 * device address: make that first call (or set CUDA_MODULE_LOADING=EAGER)
 * before reserving the rest of the device's memory.  Limits: num_parts k <=
 * 16384 (JET_ERR_INVALID beyond), part ids must lie in [0, k).  Every call
 * shares the array, so calls that overlap on the GPU (different streams, no
 * ordering between them) race and must be serialised by the caller.  Graph
 * arrays and part[] are device pointers; out[6] is host memory (the call waits
 * for its stream); stream NULL means the legacy default stream. */
int jet_pstat_noalloc(int tier, int64_t n, int64_t nnz, const void* row_map, const void* entries, const void* values,
                      const void* vweights, const int32_t* part, int32_t k, int64_t* out, void* stream);

/* ---------------------------------------------------------------- runtime
 * Library version string, last error message (thread-local), device sanity. */
const char* jet_version(void);
const char* jet_last_error(void);
int jet_device_ok(void);

/* Kernel-class timing with CUDA events on the launching stream (used by the
 * benchmark).  Classes: 0 table build, 1 LP select, 2 afterburner, 3 small
 * table update, 4 contraction (phase, host syncs included), 5 coarsening map
 * (phase), 6 table build of the finest level only, 7 rebalance select/score,
 * 8 rebalance sort, 9 eviction, 10 apply moves, 11 large table update,
 * 12 cut change.  Classes 1-3 and 7-12 are bracketed on levels that run on
 * the host-driven loop (set jet_set_refine_drivers(0) to run every level
 * there); their algorithmic bytes come from device-side counts of that
 * iteration.  jet_prof_read fills ms[13], bytes[13], launches[13]. */
int jet_prof_enable(int on);
/* Phase clocks of the persistent level loops (one CTA, cluster, cooperative
 * grid): with on = 1 a device buffer is cleared and the loops add, per
 * phase, the SM clock cycles their first thread spent and the number of
 * times the phase ran; on = 0 copies out[6 * 24] and stops.  Layout:
 * driver d (0 one CTA, 1 cluster, 2 cooperative) at out[48 d]: cycles of
 * phases 0-23, then their counts.  Phases: 0 LP select, 1 afterburner,
 * 2 hub afterburner, 3 rebalance prep, 4 rebalance select, 5 bucket scan,
 * 6 candidate sort, 7 eviction, 8 strong tail, 9 apply, 10 update subtract,
 * 11 update add + mark, 12 row rebuild, 13 cut change, 14 control, 15 copy,
 * 16 cookie cutter, 17 strong destinations, 18 strong re-draws, 19 sorted
 * weight prefix. */
int jet_prof_phases(int on, uint64_t* out);
int jet_prof_read(double* ms, double* bytes, int64_t* launches);

/* Number of CUDA kernels this library has launched in this process. */
int64_t jet_launch_count(void);

/* Test hooks for failure handling (no counterpart in the reference, whose
 * only failure path, a Metis error, exits the process:
 * src/initial_partition.hpp:106-109).  None faults, traps or hangs a GPU.
 *   jet_test_inject_metis_failures(count): the next `count` Metis calls of
 *     this process report METIS_ERROR without running (the partition call
 *     then returns JET_ERR_METIS); returns the previous count.
 *   jet_test_grid_barrier: one cooperative launch of `blocks` blocks that
 *     meet `rounds` times at the cooperative level driver's software grid
 *     barrier, each wait limited to 2^spin_cap_log2 polls; absent_block
 *     (or -1) never arrives.  JET_OK when every barrier completed,
 *     JET_ERR_TIMEOUT when a wait ran out; *passed = barrier passages.
 *   jet_test_table_overflow: inserts parts 0..nparts-1 into a shared-memory
 *     connectivity table of `cap` slots (k parts) with the table-build insert;
 *     JET_ERR_OVERFLOW when the probe bound flagged a full table. */
int jet_test_inject_metis_failures(int count);
/* Coarsest-graph Metis calls of this process: out[6] = {calls served by helper
 * processes, helper calls whose transfer failed (rerun in-process, the helper
 * replaced), in-process calls, helpers started, 1 if helpers could not be
 * started, helper calls on which Metis reported an error (rerun in-process
 * once)}. */
int jet_metis_call_stats(int64_t* out);
int jet_test_grid_barrier(int blocks, int absent_block, int spin_cap_log2, int rounds, int* passed);
int jet_test_table_overflow(int cap, int k, int nparts, int* claimed);

/* Device memory for callers without a CUDA toolchain of their own (the C++
 * drop-in include/jet.h uses these for the device views it allocates, as
 * Kokkos allocates the reference's View("label", n), app/driver.cpp:102).
 * jet_copy copies between any two host or device pointers (cudaMemcpyDefault). */
int jet_device_alloc(int64_t bytes, void** ptr);

int jet_device_free(void* ptr);
int jet_copy(void* dst, const void* src, int64_t bytes);

/* METIS text graph reader with the reference's rules (app/io.hpp:99-217),
 * parsed in parallel on `threads` host threads (0 = all cores).  Allocates
 * row_map[n+1], entries[nnz] and values[nnz] in host memory in the tier's
 * integer types; release each with jet_free_host.  Unweighted files (fmt 0)
 * give unit edge weights and *uniform_ew = 1.  JET_ERR_INVALID on a
 * malformed file (message in jet_last_error()). */
int jet_read_metis(const char* path, int tier, int threads, int64_t* n, int64_t* nnz, void** row_map, void** entries,
                   void** values, int* uniform_ew);
void jet_free_host(void* ptr);

/* Level-loop drivers refinement may use, process-wide (no counterpart in the
 * reference, whose loop is always host-driven, src/jet_refiner.hpp:1094-1134).
 * Every driver gives identical partitions; the choice only changes speed.
 * A level uses the first allowed of: one CTA (n <= 2048, or <= 16384 when
 * clusters are not allowed; nnz <= 262144; k <= 256), one thread-block
 * cluster of 8-16 CTAs (n <= 65536, nnz <= 2^21, k <= 512), one cooperative
 * grid kernel (n <= 262144, nnz <= 2^22, k <= 512), a CUDA graph with
 * conditional nodes, else the host loop.  JET_DRIVER_CTA_SMEM lets the
 * one-CTA loop keep the level's mutable state in shared memory (as much of
 * it as fits); without it that state stays in global memory.
 * JET_DRIVER_REB_QUEUE lets rebalancing order only the candidates whose
 * place in their bucket decides their eviction (one block, when they fit);
 * without it every rebalance sorts all candidates.  Returns the previous
 * mask. */
enum {
    JET_DRIVER_CTA = 1,
    JET_DRIVER_COOP = 2,
    JET_DRIVER_GRAPH = 4,
    JET_DRIVER_CLUSTER = 8,
    JET_DRIVER_CTA_SMEM = 16,
    JET_DRIVER_REB_QUEUE = 32,
    JET_DRIVER_ALL = 63
};
int jet_set_refine_drivers(int mask);

#ifdef __cplusplus
}
#endif
#endif
