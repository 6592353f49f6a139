/*
 * apgar_b200 — C ABI of the B200 search backend.
 *
 * Plain pointers and sizes only.  Every entry point returns an
 * apgar_b200_status; apgar_b200_last_error() returns the detail string of the
 * calling thread's last failure.  Host buffers are ordinary (pageable or
 * pinned) memory; `*_device` entry points take device pointers and a CUDA
 * stream handle passed as void*.
 *
 * Two families of entry points:
 *
 *  A. The drop-in seam for the reference's IPlanarRouteBackend
 *     (include/apgar/gpu/planar_router.h:543-560).  Records are bit-identical
 *     to the reference V1 layouts (DeviceCompiledHeaderV1 :170-188,
 *     DeviceLayerRangeV1 :190-201, DeviceNodeV1 :203-213, DeviceRunV1 :215-223,
 *     DeviceCandidatePolicyEdgeV1 :340-348, DeviceCandidateBatchQueryV1 :352-377,
 *     DeviceCandidateBatchResultV1 :381-407, DeviceCandidateCompactPathV1
 *     :413-423).  Status codes map 1:1 onto BackendErrorCode (:475-480).
 *
 *  B. Lattice mode: dense bit-packed multi-layer lattices with vias, per-net
 *     windows and uint32 costs (no reference counterpart; the reference is
 *     planar-only and whole-board).
 */
#ifndef APGAR_B200_H_
#define APGAR_B200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define APGAR_B200_API __attribute__((visibility("default")))
#else
#define APGAR_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define APGAR_B200_ABI_VERSION 1u

/* Mirrors BackendErrorCode (planar_router.h:475-480) with 0 = success. */
typedef enum apgar_b200_status {
  APGAR_B200_OK = 0,
  APGAR_B200_UNSUPPORTED = 1,        /* BackendErrorCode::kUnsupported */
  APGAR_B200_RESOURCE_EXHAUSTED = 2, /* BackendErrorCode::kResourceExhausted */
  APGAR_B200_BACKEND_FAILURE = 3,    /* BackendErrorCode::kBackendFailure */
  APGAR_B200_INTERNAL_INVARIANT = 4  /* BackendErrorCode::kInternalInvariant */
} apgar_b200_status;

/* Per-query outcome; values 0..3 equal KernelCompletion (planar_router.h:294-299). */
enum {
  APGAR_B200_COMPLETION_REACHED = 0,
  APGAR_B200_COMPLETION_DISCONNECTED = 1,
  APGAR_B200_COMPLETION_BUDGET_EXHAUSTED = 2,
  APGAR_B200_COMPLETION_CANCELLED = 3,
  /* lattice mode only: the net was not admitted (cost domain, width or path
   * arena bound) and carries no result */
  APGAR_B200_COMPLETION_REJECTED = 4
};

#define APGAR_B200_UNREACHABLE 0xFFFFFFFFu

APGAR_B200_API uint32_t apgar_b200_abi_version(void);

/* Copies the calling thread's last error detail (NUL-terminated, truncated to
 * capacity) and returns its full length. */
APGAR_B200_API size_t apgar_b200_last_error(char* buffer, size_t capacity);

/* Replaces BackendMetadata discovery (planar_router.h:281-292,
 * gpu/cuda/planar_router.cu:2006-2046) for the current CUDA device. */
typedef struct apgar_b200_metadata {
  char device_name[256];
  char device_uuid[40];
  uint32_t compute_capability_major;
  uint32_t compute_capability_minor;
  uint32_t runtime_version;
  uint32_t driver_version;
  uint64_t global_memory_bytes;
  uint32_t multiprocessor_count;
  uint32_t reserved;
} apgar_b200_metadata;

APGAR_B200_API int apgar_b200_query_metadata(apgar_b200_metadata* out);

/* ======================= B. lattice mode ======================= */

typedef struct apgar_b200_lattice_desc {
  int32_t layers;          /* 1..8 */
  int32_t height, width;   /* width is a multiple of 32 */
  const uint32_t* blocked; /* host: [layers][height][width/32], bit x%32 of word x/32 */
  const uint32_t* via_ok;  /* host: [layers-1][height][width/32] or NULL (all vias allowed) */
  uint32_t orth, diag, via;
} apgar_b200_lattice_desc;

typedef struct apgar_b200_lattice_net {
  uint32_t start_layer, start_x, start_y;
  uint32_t goal_layer, goal_x, goal_y;
  uint32_t win_x0, win_y0, win_w, win_h; /* window in lattice cells, all layers */
} apgar_b200_lattice_net;

typedef struct apgar_b200_lattice_result {
  uint32_t cost;         /* APGAR_B200_UNREACHABLE unless reached */
  uint32_t completion;   /* APGAR_B200_COMPLETION_* */
  uint32_t sweeps;       /* row sweeps executed (including the final quiet one) */
  uint32_t path_len;     /* cells in the reverse path (goal first) */
  uint64_t path_offset;  /* into the packed path array */
  uint64_t arena_offset; /* internal staging offset; zero once results are packed */
  uint32_t row_steps;    /* window rows processed (all layers of a row = 1) */
  uint32_t row_stores;   /* layer rows written back */
  uint32_t row_loads;    /* layer rows read (current and re-read predecessor rows) */
  uint32_t reserved;
} apgar_b200_lattice_result;

/* Uploads the lattice masks to the current device (the prepared view). */
APGAR_B200_API int apgar_b200_lattice_upload(const apgar_b200_lattice_desc* desc, void** out_lattice);
APGAR_B200_API int apgar_b200_lattice_release(void* lattice);

/* End-to-end batch on host buffers: copies the nets in, searches every net in
 * its window, and copies results and packed reverse paths (global cell ids
 * (layer*height + y)*width + x, goal first) out.  `paths` may be NULL to skip
 * the path copy; *path_total receives the number of path cells.  `cancel`
 * (optional) is polled between sweeps; non-zero cancels unfinished nets. */
APGAR_B200_API int apgar_b200_lattice_route(void* lattice, const apgar_b200_lattice_net* nets, uint32_t count,
                             uint32_t max_sweeps, const volatile uint32_t* cancel,
                             apgar_b200_lattice_result* results, uint32_t* paths,
                             uint64_t path_capacity, uint64_t* path_total);

/* Resident form for repeated launches: plan once (host planning, workspace
 * allocation, nets copied to the device), then execute on a stream (launches
 * only; capturable in a CUDA graph), then read back. */
APGAR_B200_API int apgar_b200_lattice_plan(void* lattice, const apgar_b200_lattice_net* nets, uint32_t count,
                            uint32_t max_sweeps, void** out_plan);
APGAR_B200_API int apgar_b200_lattice_execute(void* plan, void* stream);
APGAR_B200_API int apgar_b200_lattice_readback(void* plan, apgar_b200_lattice_result* results, uint32_t* paths,
                                uint64_t path_capacity, uint64_t* path_total);
/* Device pointers of the plan's result records and packed paths. */
APGAR_B200_API int apgar_b200_lattice_device_results(void* plan, const apgar_b200_lattice_result** results,
                                      const uint32_t** paths);
typedef struct apgar_b200_plan_info {
  uint32_t net_count;
  uint32_t kernel_launches;     /* launches per execute */
  uint32_t class_count;         /* width classes launched */
  uint32_t reserved;
  uint64_t workspace_bytes;     /* label slabs + arena + records */
  uint64_t label_cells;         /* sum of layers*rows*pitch over nets */
  uint64_t path_arena_capacity; /* cells */
} apgar_b200_plan_info;
APGAR_B200_API int apgar_b200_lattice_plan_info(void* plan, apgar_b200_plan_info* out);
APGAR_B200_API int apgar_b200_lattice_plan_release(void* plan);

#ifdef __cplusplus
}
#endif

#endif /* APGAR_B200_H_ */
