/* libccs: B200-native optimal 3x3 cube solving (half-turn metric) behind a C ABI.
 *
 * The library replaces the reference's kernel boundary: src/cuda_cube_solver/device.py:115-141
 * (module(*defines) -> CuPy RawModule of kernels.cu, DeviceTables) and the kernel launches at
 * solver.py:238-240,302 and table.py:72-79,103,115,118,136.  Host buffers are borrowed for the
 * duration of a call; the library owns all device memory behind a handle.  Every call returns 0
 * or a negative CCS_E_* code; ccs_last_error() gives the message of the last failure on the
 * calling thread.  A handle is not reentrant: use one handle per host thread (the server entry
 * points are the exception, see below).
 *
 * Packed state: 5 little-endian uint32 words, corner bytes cp | co << 3 (positions 0..7), edge
 * bytes ep | eo << 4 (positions 0..11) -- the reference's device.pack_states (device.py:144-148).
 * Moves are numbered 0..17 = U U2 U' R R2 R' F F2 F' D D2 D' L L2 L' B B2 B' (cubie.py:115-124).
 */
#ifndef CCS_H
#define CCS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CCS_OK 0
#define CCS_E_CUDA (-1)       /* a CUDA call failed */
#define CCS_E_NOMEM (-2)      /* device or host allocation failed */
#define CCS_E_ARG (-3)        /* bad argument: unknown kind / format, bad size (ValueError) */
#define CCS_E_FILE (-4)       /* table file missing, unreadable or of the wrong size */
#define CCS_E_CHECK (-5)      /* a self-check failed (AssertionError in the reference) */
#define CCS_E_UNREACHABLE (-6)/* BFS found entries unreachable (RuntimeError in the reference) */
#define CCS_E_STATE (-7)      /* call not valid in this state (no table loaded, server stopped) */
#define CCS_E_TIMEOUT (-8)    /* a bounded wait ran out */

#define CCS_FMT_BLOCK 0       /* 2-bit block table, "prune-ud-<kind>-blk.bin" */
#define CCS_FMT_B3 1          /* base-3 block table, "prune-ud-<kind>-b3.bin" */
#define CCS_FMT_MOD3 2        /* the reference's mod-3 file "prune-ud-<kind>.bin": depth mod 3 in  */
                              /*   two bits, sixteen entries per little-endian uint32, 3 past the   */
                              /*   end (table.py:82-129,140-167); written by builds, not solved on  */

typedef struct ccs_handle ccs_handle;

typedef void (*ccs_log_fn)(const char* message);

/* Library version, (major << 16) | minor. */
int ccs_version(void);

/* Message of the last failure on this thread ("" if none). */
const char* ccs_last_error(void);

/* Free and total memory of a device (kinds.pick, kinds.py:198-211, reads cudaMemGetInfo). */
int ccs_mem_info(int device, uint64_t* free_bytes, uint64_t* total_bytes);

/* Number of SMs of a device. */
int ccs_device_sms(int device, int* sms);

/* Open / close a handle on a device (replaces DeviceTables construction, device.py:125-141). */
int ccs_open(int device, ccs_handle** out);
int ccs_close(ccs_handle* h);

/* Table kind by name: "304" or a group kind "s4", "d4f", "a4t", "d4t", "d4", "a4"
 * (kinds.get, kinds.py:100-105).  Writes the E-content class count and the number of entries. */
int ccs_kind_info(const char* kind, int* nec, uint64_t* n_entries);

/* A custom group kind from generators (kinds.GroupKind, kinds.py:56-96): n_gens pairs of
 * perm[4] and flips[4].  Registers it under `name` for the other calls.  Returns CCS_E_ARG with
 * "<name>: group not normalised by the UD symmetries; ..." when symmetry reduction would be wrong. */
int ccs_register_group_kind(const char* name, int n_gens, const int32_t* perms, const int32_t* flips);

/* Constant tables of a kind (for cross-checks): corner classidx[153090], class_rep[9930],
 * class_stab[9930], gen_class[384], gen_rep[2*384]; any pointer may be NULL. */
int ccs_kind_tables(const char* kind, uint32_t* classidx, uint32_t* class_rep, uint16_t* class_stab,
                    uint16_t* gen_class, uint16_t* gen_rep);

/* Select the table kind used by ccs_index / ccs_unrank without loading a table. */
int ccs_set_kind(ccs_handle* h, const char* kind);

/* Load a solving table file into device memory (table.load_device, table.py:28-38; size checked
 * against the kind and format like table.py:36-37).  Replaces any table already loaded. */
int ccs_load_table(ccs_handle* h, const char* kind, int format, const char* path);

/* Build a table on the device (table.generate + build_preset, table.py:82-129,170-200): exact
 * BFS, histogram self-check, encode in `format`.  If out_path is not NULL the solving file is
 * written there (through "<out_path>.tmp" and a rename).  If keep_resident, the solving table
 * stays loaded in the handle as if ccs_load_table had been called (keep_resident = 2: it becomes
 * the second table, see ccs_attach_table; with keep_resident = 0 a table already loaded keeps
 * its kind, on success and on failure).  depth_counts receives up to
 * max_depths per-depth entry counts, n_depths their number; seconds the build time (GPU work,
 * without the file write).  log may be NULL. */
int ccs_build_table(ccs_handle* h, const char* kind, int format, const char* out_path, int keep_resident,
                    uint64_t* depth_counts, int max_depths, int* n_depths, double* seconds, ccs_log_fn log);

/* One BFS, several files (table.build, table.py:140-167, which writes the mod-3 and block files
 * of one generate): each non-NULL path is written from the same exact-depth array, through
 * "<path>.tmp" and a rename.  The handle's resident tables are left as they are, and so is the
 * kind they were loaded with.  Counts, seconds and log as for ccs_build_table. */
int ccs_build_table_files(ccs_handle* h, const char* kind, const char* block_path, const char* b3_path,
                          const char* mod3_path, uint64_t* depth_counts, int max_depths, int* n_depths,
                          double* seconds, ccs_log_fn log);

/* Base-3 file from the mod-3 and block files of `kind` (table.build_b3_table and write_b3,
 * table.py:52-79): both are read onto the device (sizes checked), encoded there, and the base-3
 * file is written to b3_path (through "<b3_path>.tmp").  The handle's tables are untouched. */
int ccs_encode_b3_file(ccs_handle* h, const char* kind, const char* mod3_path, const char* block_path,
                       const char* b3_path);

/* Write a resident table -- table 0, or 1 for the second table -- to a file in chunks through
 * pinned staging (table.save_device, table.py:20-25), through "<path>.tmp" and a rename. */
int ccs_save_table(ccs_handle* h, int table, const char* path);

/* Entries of a resident table (0, or 1 for the second) per stored lower bound, counted on the
 * device: bins[v] = entries whose decoded value is v, the last bin also holding larger values
 * (table.histogram, table.py:132-137, counts the mod-3 table's four values; the solving tables
 * hold a bound per entry, so the bins are those bounds: exact below a 2-bit block's minimum + 3,
 * and "at least" at the cut of either format).  The bins sum to the kind's entry count. */
int ccs_table_histogram(ccs_handle* h, int table, uint64_t* bins, int n_bins);

/* One BFS pass of the last ccs_build_table: the depth it assigned, forward (1: expand the
 * frontier, kernels.cu:544-574) or backward (0: unvisited entries test their neighbours,
 * kernels.cu:577-611), the entries found, the random depth-byte reads and the claim attempts
 * (atomics) it made, and its device time.  Algorithmic bytes of a pass: one sequential scan of
 * the depth bytes plus one 32-byte sector per random read and per claim. */
typedef struct ccs_bfs_pass {
    int32_t depth;
    int32_t forward;
    uint64_t found;
    uint64_t random_reads;
    uint64_t claims;
    double seconds;
} ccs_bfs_pass;
int ccs_last_build_passes(ccs_handle* h, ccs_bfs_pass* out, int max_out, int* n_out);

/* A second resident table (table id 1) of the same kind family and format as the first, e.g. d4
 * next to d4t: one search launch then serves cubes of either table, chosen per cube.  Loaded from
 * a file here; ccs_build_table with keep_resident = 2 builds it in place instead. */
int ccs_attach_table(ccs_handle* h, const char* kind, int format, const char* path);

/* Copy the loaded solving table (n_bytes = its size) to host memory. */
int ccs_table_bytes(ccs_handle* h, uint64_t* n_bytes);
int ccs_table_copy(ccs_handle* h, void* dst, uint64_t n_bytes);

/* Index of packed states under the loaded kind (the reference's probe_index kernel,
 * kernels.cu:626-642): move >= 0 right-multiplies by that move first, move <= -2 left-multiplies
 * by move -2 - move, -1 leaves the state.  out_idx[n], out_states[n*5] (may be NULL). */
int ccs_index(ccs_handle* h, const uint32_t* states, int n, int move, uint64_t* out_idx, uint32_t* out_states);

/* Representative state of each index (the reference's unrank, kernels.cu:294-379). */
int ccs_unrank(ccs_handle* h, const uint64_t* idx, int n, uint32_t* out_states);

/* Table lower bound of packed states (probe_block, kernels.cu:737-746). */
int ccs_lower_bound(ccs_handle* h, const uint32_t* states, int n, uint32_t* out);

/* Root bounds of cubes: the six frames' lower bounds (GpuSolver.root_h, solver.py:226-252). */
int ccs_root_bounds(ccs_handle* h, const uint32_t* states, int n, uint32_t* out_h6);

typedef struct ccs_solve_opts {
    int base_plen;            /* prefix length of a cube's first iterations (reference: 4) */
    double deeper_at0;        /* an iteration of >= this many nodes makes the next one use a */
    double deeper_at1;        /*   prefix one move longer (reference: 5e7, 3e9); see also     */
                              /*   few_divisor                                                */
    int blocks_per_sm;        /* persistent grid = blocks_per_sm * SMs (0: default)         */
    int threads;              /* threads per block: 128, 256 or 512 (0: default)            */
    double timeout_s;         /* give up after this long (0: no limit)                      */
    int spread;               /* lanes work on up to this many queued cubes at once (0: 4096) */
    int variant;              /* search kernel: 0 automatic (2 below 64 cubes, else 3), 1 = 256 */
                              /*   threads x 2 blocks/SM, 2 = sibling lookahead (two probe      */
                              /*   chains per lane), 3 = 256 x 3, 6 = 128 x 4, 7 = 512 x 1,      */
                              /*   8 = lookahead 256 x 3 (4-5: loop-control forms)              */
    double shallow_at0;       /* an iteration of < this many nodes makes the next one use a    */
    double shallow_at1;       /*   prefix one move shorter (0: 1e5 / 1.5e6, < 0: off)          */
    int move_min;             /* lanes waiting before a frame-update pass runs (0: 8; 1 in a   */
                              /*   ccs_solve of fewer than 64 cubes)                            */
    int move_age;             /* warp iterations a lane may wait for it (0: 4)                 */
    int probe_min;            /* a warp keeps probing (pruned children -> next sibling) while  */
                              /*   at least this many lanes have a probe (0: 16, or 8 in a      */
                              /*   ccs_solve of fewer than 64 cubes; > 32: off)                 */
    int steal;                /* work stealing: lanes donate unexplored subtrees to idle lanes  */
                              /*   (phase-ordered variants; 0 or 1: on, asked for by any idle   */
                              /*   lane; 2: on, asked for by whole idle warps; < 0: off).  The  */
                              /*   server takes 0 as 2 (whole idle warps ask).                  */
    int steal_depth;          /* a donated node's slack -- moves to the bound beyond its largest */
                              /*   frame bound -- is at least this (0: 2)                       */
    int steal_period;         /* a lane with work checks for starving lanes every this many    */
                              /*   iterations, a power of two (0: 64)                           */
    int steal_target;         /* donors stop once this many subtrees wait (0: 512)              */
    int few_divisor;          /* while at most 4 cubes are in flight, deeper_at0/1 are divided */
                              /*   by this (0: 50, or 200 in a ccs_solve of fewer than 64       */
                              /*   cubes; 1: never, the reference's plain thresholds)           */
    double steal_min_nodes;   /* subtrees of a cube are donated only once its previous          */
                              /*   iteration reached this many nodes (0: 1e7; < 0: always)      */
    int rotate;               /* a live entry at the work ring's head moves to the tail once   */
                              /*   the queue spans half of `spread` (1), or half the ring (-1), */
                              /*   so every queued cube stays within the lanes' scan window     */
                              /*   (0: 1 for the server, -1 for ccs_solve)                      */
} ccs_solve_opts;

typedef struct ccs_result {
    int32_t status;           /* 0 solved, < 0 error */
    int32_t length;           /* optimal length in half-turn moves */
    uint8_t moves[24];        /* the solution, `length` moves */
    uint64_t nodes;           /* children generated over all iterations */
    uint64_t probes;          /* table lookups */
    double seconds;           /* admission to solution, device clock */
    uint64_t iter_nodes[24];  /* nodes per IDA* bound (Solution.iteration_nodes) */
} ccs_result;

/* Solve n cubes together (GpuSolver.solve, solver.py:254-320): one persistent launch advances
 * every cube through its IDA* bounds on the device.  results[n]; n < 1,048,575 per call. */
int ccs_solve(ccs_handle* h, const uint32_t* states, int n, const ccs_solve_opts* opts, ccs_result* results);

/* ccs_solve with a table per cube: table_ids[n] of 0 (the first table) or 1 (the attached one). */
int ccs_solve_tables(ccs_handle* h, const uint32_t* states, const uint8_t* table_ids, int n,
                     const ccs_solve_opts* opts, ccs_result* results);

/* ccs_solve without any allocation, for callers that cannot allocate device memory while they
 * solve: a process whose GPU memory is owned by a caching pool or a framework's allocator (its
 * own cudaMalloc would fail or fragment the pool), or a service that fixes its memory footprint
 * at start-up.  No counterpart in the reference.  The search buffers are one fixed array in the
 * library's device image (304 KB on every GPU that loads the library); at most
 * CCS_NOALLOC_MAX_CUBES cubes per call, prefixes of at most 4 moves (opts->base_plen <= 4;
 * deeper_at0/1 are ignored), the first table only, devices 0..15.  The first call on a device sets
 * the array up (with that device current) and should come before any stream capture; a call after
 * a device reset sets it up again.  One array per process and device, shared by every handle on
 * that device: calls on one device would race on it, so the library runs them one at a time (a
 * per-device lock; calls on different devices do not wait for each other). */
#define CCS_NOALLOC_MAX_CUBES 256
int ccs_solve_noalloc(ccs_handle* h, const uint32_t* states, int n, const ccs_solve_opts* opts,
                      ccs_result* results);

/* Device time of the last ccs_solve's search kernels (ms) and its total table probes. */
int ccs_last_solve_stats(ccs_handle* h, double* kernel_ms, uint64_t* probes, int* launches);

/* Bytes the last ccs_solve copied host -> device (cube slots, admission entries, queue state) and
 * device -> host (queue state after each launch, cube slots). */
int ccs_last_solve_io_bytes(ccs_handle* h, uint64_t* h2d, uint64_t* d2h);

/* Subtrees the last ccs_solve's lanes donated to idle lanes (work stealing; no counterpart in the
 * reference, whose work items are fixed per bound, solver.py:189-195). */
int ccs_last_solve_donations(ccs_handle* h, uint64_t* donated);

/* Random 32-byte sector gather ceiling of a device (the table probes' memory roofline): random
 * sector loads from a `bytes` buffer, 8 in flight per thread; sectors_per_s and the time. */
int ccs_gather_bench(int device, uint64_t bytes, int rounds, double* sectors_per_s, double* ms);

/* The probe step alone on the loaded table (random states: index + lower bound, no search
 * control), for comparison with the search kernel's probe rate. */
int ccs_probe_bench(ccs_handle* h, int n_states, int rounds, double* probes_per_s, double* ms);

/* ---- server: continuous batching (thread-safe against each other) -------------------------
 * ccs_server_start runs a service thread that owns a persistent search launch over `slots`
 * cube slots; ccs_server_submit queues a cube (returns a request id), ccs_server_poll returns
 * up to max_out finished results with their request ids.  Cubes that arrive while others are on
 * the GPU are admitted into free slots without waiting for the running ones.  slots <
 * 1,048,575; each takes 456 bytes of device memory (cube slot and ring positions). */
int ccs_server_start(ccs_handle* h, int slots, const ccs_solve_opts* opts);

/* ccs_server_start with admission by device memory (continuous batching; the reference has fixed
 * --batch chunks only, __main__.py:129-133): the server holds a fixed footprint --
 * resident tables, constants, prefix lists, queue state, work-stealing cells and the persistent
 * launch's per-lane search stacks -- plus 456 bytes per cube in flight (its slot, ring positions
 * and admission entry); a cube is admitted only while the total stays within budget_bytes.
 * CCS_E_NOMEM if the fixed footprint alone exceeds the budget.  slots_out (may be NULL): the cubes
 * the budget admits at once (at most 65,536). */
int ccs_server_start_budget(ccs_handle* h, uint64_t budget_bytes, const ccs_solve_opts* opts, int* slots_out);

/* The running server's budget (0: none), fixed footprint and bytes per cube in flight (bytes), and
 * the most cubes it has held in flight at once. */
int ccs_server_memory(ccs_handle* h, uint64_t* budget, uint64_t* fixed, uint64_t* per_cube, uint64_t* peak_in_flight);
int ccs_server_submit(ccs_handle* h, const uint32_t* state, uint64_t* request_id);
int ccs_server_submit_table(ccs_handle* h, const uint32_t* state, int table_id, uint64_t* request_id);
int ccs_server_poll(ccs_handle* h, int max_out, uint64_t* request_ids, ccs_result* results, int* n_out);
int ccs_server_stop(ccs_handle* h);

#ifdef __cplusplus
}
#endif

#endif /* CCS_H */
