/*
 * ccs_cuda.h -- C ABI of the B200 (sm_100a) Catmull-Clark refinement library.
 *
 * Drop-in for the refinement entry points of jdupuy/HalfedgeCatmullClark's
 * CatmullClark.h.  The library keeps the reference's data layout: a
 * `cc_Mesh` cage goes in, a `cc_Subd` with the packed level-by-level
 * halfedge / crease / vertex-point arrays comes out, byte-compatible with
 * the reference's accessors (ccs_HalfedgeTwinID, ccs_VertexPoint, ...).
 * Each `_cuda` function replaces the reference function of the same name
 * without the suffix; the work runs as CUDA kernels on the GPU that is
 * current when `ccs_Create_cuda` is called, and results reach the host
 * arrays of the `cc_Subd` by `ccs_Download_cuda`.
 *
 * Differences from the reference, all deliberate:
 *   - functions return a status (CCS_OK = 0) instead of void / aborting;
 *     C code that ignores the result still compiles unchanged;
 *   - a subd made by ccs_Create_cuda must be released by ccs_Release_cuda;
 *   - the host arrays of such a subd are written only by ccs_Download_cuda.
 *
 * Thread safety: calls on one subd must not overlap; distinct subds are
 * independent.  Each subd owns one CUDA stream (replaceable with
 * ccs_SetStream_cuda); every call is stream-ordered on it and the refine
 * calls return without waiting for the GPU.
 *
 * Include CatmullClark.h before this header to share its type definitions;
 * otherwise this header defines the same types with the same layout.
 */
#ifndef CCS_CUDA_H
#define CCS_CUDA_H

#include <stdint.h>
#include <stddef.h>
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef CC_INCLUDE_CC_H
#define CC_INCLUDE_CC_H
/* Types of CatmullClark.h:17-71 and :136-142, same members and layout. */
typedef union { struct { float x, y, z; }; float array[3]; } cc_VertexPoint;
typedef union { struct { float u, v; }; float array[2]; } cc_VertexUv;
typedef struct { int32_t nextID; int32_t prevID; float sharpness; } cc_Crease;
typedef struct {
    int32_t twinID, nextID, prevID, faceID, edgeID, vertexID, uvID;
} cc_Halfedge;
typedef struct {
    int32_t twinID;
    int32_t edgeID;
    int32_t vertexID;
#ifndef CC_DISABLE_UV
    int32_t uvID;
#endif
} cc_Halfedge_SemiRegular;
typedef struct {
    int32_t vertexCount;
    int32_t uvCount;
    int32_t halfedgeCount;
    int32_t edgeCount;
    int32_t faceCount;
    int32_t *vertexToHalfedgeIDs;
    int32_t *edgeToHalfedgeIDs;
    int32_t *faceToHalfedgeIDs;
    cc_VertexPoint *vertexPoints;
    cc_VertexUv *uvs;
    cc_Halfedge *halfedges;
    cc_Crease *creases;
} cc_Mesh;
typedef struct {
    const cc_Mesh *cage;
    cc_VertexPoint *vertexPoints;
    cc_Halfedge_SemiRegular *halfedges;
    cc_Crease *creases;
    int32_t maxDepth;
} cc_Subd;
#endif /* CC_INCLUDE_CC_H */

/* Status codes.  The reference aborts through CC_ASSERT (CatmullClark.h:
 * 227-230) or returns NULL; this library returns one of these instead. */
enum {
    CCS_OK = 0,
    CCS_ERR_ARG = -1,          /* NULL / inconsistent argument            */
    CCS_ERR_ALLOC = -2,        /* host or device allocation failed        */
    CCS_ERR_OVERFLOW = -3,     /* a count at this depth exceeds int32     */
    CCS_ERR_CUDA = -4,         /* a CUDA call failed                      */
    CCS_ERR_TIMEOUT = -5,      /* a bounded device wait gave up           */
    CCS_ERR_STATE = -6,        /* call order (e.g. points before topology) */
    CCS_ERR_UNSUPPORTED = -7,  /* option not available for this layout     */
    CCS_ERR_SCRATCH_LIMIT = -8 /* problem larger than a fixed scratch area */
};

/* Flags for ccs_CreateEx_cuda / ccs_SetFlags_cuda. */
enum {
    CCS_FLAG_NO_UV = 1u << 0,          /* 12-byte halfedge records (the
                                          CC_DISABLE_UV build of the record) */
    CCS_FLAG_PAGEABLE_HOST = 1u << 1,  /* host arrays from malloc, not pinned */
    CCS_FLAG_DETERMINISTIC = 1u << 2,  /* scatter points summed per vertex in
                                          increasing halfedge order (the
                                          reference's one-thread order: bit-
                                          identical) instead of float atomics */
    CCS_FLAG_NO_GRAPH = 1u << 3,       /* launch kernels one by one instead
                                          of replaying a captured CUDA graph  */
    CCS_FLAG_SEPARATE_PASSES = 1u << 4 /* run the reference's pass structure
                                          (no per-level kernel fusion)        */
};

/* ---------------------------------------------------------------------- */
/* Construction / destruction                                              */
/* ---------------------------------------------------------------------- */

/* Replaces ccs_Create (CatmullClark.h:145, :953-970).  Allocates the host
 * arrays of the returned subd (pinned) and their device mirrors, uploads the
 * cage.  The cage is borrowed and must outlive the subd.  Returns NULL on
 * failure; ccs_LastError_cuda() tells why.  16-byte records (with uvID). */
cc_Subd *ccs_Create_cuda(const cc_Mesh *cage, int32_t maxDepth);

/* ccs_Create_cuda with CCS_FLAG_* options; *out receives the subd. */
int ccs_CreateEx_cuda(const cc_Mesh *cage, int32_t maxDepth, uint32_t flags, cc_Subd **out);

/* Replaces ccs_Release (CatmullClark.h:146, :977-983). NULL is a no-op. */
void ccs_Release_cuda(cc_Subd *subd);

/* `.ccm` cage files.  ccs_LoadCage_cuda replaces ccm_Load (CatmullClark.h:
 * 74, :3186-3220): the cage and all its arrays land in one page-locked host
 * allocation, so ccs_Create_cuda uploads it by DMA straight from the file's
 * buffer; NULL on failure (ccs_LastError_cuda: CCS_ERR_ARG for a missing or
 * malformed file).  Release it with ccs_ReleaseCage_cuda (ccm_Release, :79),
 * after every subd made from it.  ccs_SaveCage_cuda replaces ccm_Save
 * (:80, :3227-3269) and writes the same bytes (header padding zeroed). */
cc_Mesh *ccs_LoadCage_cuda(const char *path);
void ccs_ReleaseCage_cuda(cc_Mesh *cage);
int ccs_SaveCage_cuda(const cc_Mesh *cage, const char *path);

/* A polygon mesh: what the reference's OBJ converter reads (examples/
 * obj_to_ccm.c LoadObj :666-752), as arrays.  Face f's corners are
 * faceOffsets[f] .. faceOffsets[f + 1] - 1 (faceOffsets[0] = 0) of
 * faceVertices (0-based vertex IDs) and of faceUvs (0-based texture IDs, or
 * NULL: every uvID 0, as LoadObj for faces without `vt`).  creaseVertices
 * holds creaseTagCount pairs (v0, v1) with creaseSharpness[t]: the
 * `t crease 2/1/0 v0 v1 s` tags.  Arrays may be host or device memory. */
typedef struct {
    int32_t vertexCount, uvCount, faceCount, creaseTagCount;
    const int32_t *faceOffsets;
    const int32_t *faceVertices;
    const int32_t *faceUvs;
    const float *vertexPoints;   /* vertexCount x 3 */
    const float *uvs;            /* uvCount x 2 */
    const int32_t *creaseVertices;
    const float *creaseSharpness;
} ccs_PolygonMesh;

/* Builds the halfedge cage of `mesh` on the GPU -- twins, edge, vertex and
 * face maps, creases, boundary sharpness 16 and crease chains, numbered as
 * LoadObj numbers them (obj_to_ccm.c:88-450, :538-561) -- into one
 * page-locked block like ccs_LoadCage_cuda's (release it with
 * ccs_ReleaseCage_cuda).  CCS_ERR_ARG for a face with fewer than 3 corners
 * or two consecutive corners on one vertex, an index out of range, or a
 * directed edge used twice.  Waits for the GPU before returning. */
int ccs_BuildCage_cuda(const ccs_PolygonMesh *mesh, cc_Mesh **out, void *stream);

/* ---------------------------------------------------------------------- */
/* Refinement (CatmullClark.h:197-212)                                     */
/* ---------------------------------------------------------------------- */
int ccs_Refine_Scatter_cuda(cc_Subd *subd);                   /* :198, :3060 */
int ccs_Refine_Gather_cuda(cc_Subd *subd);                    /* :199, :3066 */
int ccs_RefineVertexPoints_Gather_cuda(cc_Subd *subd);        /* :200, :2659 */
int ccs_RefineVertexPoints_Scatter_cuda(cc_Subd *subd);       /* :201, :2631 */
int ccs_RefineHalfedges_cuda(cc_Subd *subd);                  /* :202, :2803 */
int ccs_RefineCreases_cuda(cc_Subd *subd);                    /* :203, :3033 */
int ccs_RefineVertexUvs_cuda(cc_Subd *subd);                  /* :205, :2928 */
int ccs_Refine_NoCreases_Gather_cuda(cc_Subd *subd);          /* :209, :3078 */
int ccs_Refine_NoCreases_Scatter_cuda(cc_Subd *subd);         /* :210, :3072 */
int ccs_RefineVertexPoints_NoCreases_Gather_cuda(cc_Subd *subd);   /* :211, :2672 */
int ccs_RefineVertexPoints_NoCreases_Scatter_cuda(cc_Subd *subd);  /* :212, :2645 */

/* ---------------------------------------------------------------------- */
/* Host <-> device                                                         */
/* ---------------------------------------------------------------------- */

/* Copies the device halfedges, creases and points into subd->halfedges,
 * subd->creases and subd->vertexPoints, then waits for the copy.  After it
 * the reference's accessors (CatmullClark.h:986-1395) read the results. */
int ccs_Download_cuda(cc_Subd *subd);

/* Uploads new cage points (V0 records) -- NULL re-reads subd->cage. */
int ccs_UploadCagePoints_cuda(cc_Subd *subd, const cc_VertexPoint *points);

/* Stream control.  `stream` is a cudaStream_t (NULL = the legacy default
 * stream).  The subd does not take ownership of a stream set this way. */
int ccs_SetStream_cuda(cc_Subd *subd, void *stream);
void *ccs_GetStream_cuda(const cc_Subd *subd);
int ccs_Synchronize_cuda(cc_Subd *subd);
int ccs_SetFlags_cuda(cc_Subd *subd, uint32_t flags);
uint32_t ccs_GetFlags_cuda(const cc_Subd *subd);

/* Device addresses of the subd's arrays (same layout as the host arrays). */
typedef struct {
    void *halfedges;          /* cumH records of 16 (or 12) bytes            */
    cc_Crease *creases;       /* cumC records                                */
    float *vertexPoints;      /* cumV x 3 floats                             */
    float *cagePoints;        /* V0 x 3 floats                               */
    int64_t halfedgeCount, creaseCount, vertexCount;
    int32_t recordBytes;      /* 16, or 12 with CCS_FLAG_NO_UV               */
} ccs_DeviceArrays;
int ccs_GetDeviceArrays_cuda(const cc_Subd *subd, ccs_DeviceArrays *out);

/* ---------------------------------------------------------------------- */
/* Points from caller-owned device buffers (no reference counterpart: the   */
/* building blocks of the PyTorch extension's autograd function).           */
/* ---------------------------------------------------------------------- */

/* Point modes. */
enum { CCS_POINTS_SCATTER = 0, CCS_POINTS_GATHER = 1,
       CCS_POINTS_NOCREASES_SCATTER = 2, CCS_POINTS_NOCREASES_GATHER = 3 };

/* Refines `cagePoints` (V0 x 3 floats, device) through the subd's device
 * topology into `points` (cumV x 3 floats, device) on `stream`.  The
 * topology must have been refined (ccs_RefineHalfedges_cuda and
 * ccs_RefineCreases_cuda, or a ccs_Refine_* call). */
int ccs_RefinePointsDevice_cuda(cc_Subd *subd, const float *cagePoints, float *points,
                                int mode, void *stream);

/* Adjoint of the scatter point rule: given dL/dpoints (cumV x 3, device),
 * writes dL/dcagePoints (V0 x 3, device).  Runs the transposed face, edge
 * and vertex rules as gathers, deepest level first.  Uses a scratch buffer
 * of cumV x 3 floats that the library allocates on first use and keeps. */
int ccs_AdjointPointsDevice_cuda(cc_Subd *subd, const float *gradPoints, float *gradCage,
                                 void *stream);

/* ccs_AdjointPointsDevice_cuda for callers that must not allocate GPU memory.
 * No counterpart in the reference (which has no adjoint).
 *
 * ccs_AdjointPointsDevice_cuda allocates its working buffer with cudaMalloc
 * on first use.  Some callers cannot allow that: code that is recording a
 * CUDA graph through stream capture (cudaMalloc is not allowed while a
 * stream is being captured), applications whose device memory is owned by
 * their own pool allocator (PyTorch's caching allocator, a renderer's arena)
 * and would be fragmented or overcommitted by allocations behind their
 * back, and real-time loops that forbid allocation after start-up.  This
 * entry point allocates nothing: its working buffer is a fixed array of
 * 16 MiB (4,194,304 floats) compiled into the library, which every GPU that
 * loads the library holds until the process exits.  It therefore accepts
 * subds whose refined points fit: 3 * (total refined points) <= 4,194,304,
 * i.e. at most 1,398,101 points over all levels; larger subds are refused
 * with CCS_ERR_SCRATCH_LIMIT.  The caller passes the inputs and outputs as
 * for ccs_AdjointPointsDevice_cuda.  It runs the same kernels, which sum
 * with float atomics, so the two agree up to the order of those additions
 * (within 1e-5 relative), not bit for bit.
 *
 * The first call on a device looks up that device's address of the array
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * The address is looked up again after the device's context changes (a
 * caller's cudaDeviceReset).
 * All calls share the one array, so calls whose work can overlap on the GPU
 * (different streams, or different host threads) race and must be
 * serialised by the caller. */
int ccs_AdjointPointsDeviceNoAlloc_cuda(cc_Subd *subd, const float *gradPoints, float *gradCage,
                                        void *stream);

/* The cage step of a point rule as a sparse matrix (host only; no GPU work;
 * no counterpart in the reference, whose rules it applies symbolically:
 * CatmullClark.h:1437-1463, :1602-1648 and :1872-1991 for
 * mode = CCS_POINTS_SCATTER; :1517-1548 and :1713-1756 for
 * CCS_POINTS_NOCREASES_SCATTER).  For a fixed topology and sharpness the
 * points of depth 1 are S x (cage points); rows are depth 1's points
 * ([old vertices | faces | edges]), columns cage vertices; `transpose`
 * (scatter rule only) gives S^T, the adjoint's cage level.  This is the map
 * the default pass evaluates as its cage step.  CSR arrays: rowptr (rows + 1
 * entries), col and w (nnz entries).  Call with cap = 0 for *rows and *nnz,
 * then with arrays of those sizes. */
int ccs_CageStepMatrix_cuda(const cc_Mesh *cage, int mode, int transpose, int32_t *rows, int64_t *nnz,
                            int32_t *rowptr, int32_t *col, float *w, int64_t cap);

/* Per-halfedge normals of the finest level, the refined-surface consumer of
 * the reference's GLSL library (glsl/CatmullClark_Scatter.glsl:931-960,
 * ccs_HalfedgeNormal_Fast / ccs_HalfedgeNormal): `normals` (device, H(D) x 3
 * floats) receives, per halfedge h of depth D, the normalised cross product
 * of its face's edges at h, or with `smooth` the normalised sum of those of
 * every halfedge around vertex(h) (the face normal on a boundary vertex).
 * `points` = device points of every depth as ccs_RefinePointsDevice_cuda
 * writes them, or NULL for the subd's own.  Needs the topology refined. */
int ccs_HalfedgeNormals_cuda(cc_Subd *subd, const float *points, float *normals, int smooth, void *stream);

/* Writes depth `depth` (0 = the cage) of a subd as an OBJ file with the bytes
 * of the reference's ExportToObj (examples/subd_cpu.c:22-115), formatted on
 * the GPU from the device arrays (no ccs_Download_cuda needed): "v" lines,
 * "vt" lines (per halfedge at depth >= 1; none with 12-byte records, as the
 * CC_DISABLE_UV build), "f" lines.  Waits for the subd's stream.  With
 * 16-byte records and a cage without UVs the reference prints uninitialised
 * uvIDs; here they are 0. */
int ccs_ExportObj_cuda(const cc_Subd *subd, int32_t depth, const char *path);

/* ---------------------------------------------------------------------- */
/* Batched refinement (no reference counterpart).                          */
/*                                                                         */
/* Many cages, each with its own depth, refined together: for every depth  */
/* one persistent cooperative kernel covers all cages still active at that */
/* depth, and each operation is replayed as one CUDA graph.  Every cage     */
/* keeps the single-mesh layout inside batch-wide device buffers (see      */
/* ccs_BatchCageInfo_cuda for its offsets).  Scatter rules only, 16-byte    */
/* records; every point summed in the reference's one-thread order (no      */
/* atomics), so each cage's result equals the single-mesh path bit for bit. */
/* ---------------------------------------------------------------------- */
typedef struct ccs_Batch ccs_Batch;
typedef struct {
    void *halfedges;          /* all cages' records (16 B)                   */
    cc_Crease *creases;
    float *points;            /* refined points, all cages, all depths       */
    float *cagePoints;        /* input cage points, all cages                */
    float *gradPoints;        /* adjoint input (consumed by the adjoint)     */
    float *gradCagePoints;    /* adjoint output                              */
    int64_t halfedgeCount, creaseCount, pointCount, cagePointCount;
} ccs_BatchArrays;
typedef struct {
    int32_t depth;
    int64_t cagePointOffset, cagePointCount;   /* in cagePoints / gradCagePoints */
    int64_t halfedgeOffset, halfedgeCount;
    int64_t creaseOffset, creaseCount;
    int64_t pointOffset, pointCount;           /* in points / gradPoints         */
    int64_t finestPointOffset, finestPointCount;
} ccs_BatchCageInfo;

/* Uploads `count` cages (validated; each must satisfy the twin relation
 * vertex(twin(h)) == vertex(next(h))) and sizes every buffer. */
int ccs_BatchCreate_cuda(const cc_Mesh *const *cages, const int32_t *depths, int32_t count,
                         uint32_t flags, ccs_Batch **out);
void ccs_BatchRelease_cuda(ccs_Batch *batch);
/* Topology, creases, UVs and points of every cage; mode CCS_POINTS_SCATTER
 * or CCS_POINTS_NOCREASES_SCATTER. */
int ccs_BatchRefine_cuda(ccs_Batch *batch, int mode);
/* Points only, from the batch's cagePoints buffer (topology refined before). */
int ccs_BatchRefinePoints_cuda(ccs_Batch *batch, int mode);
/* Adjoint of the scatter rule: gradPoints (consumed) -> gradCagePoints. */
int ccs_BatchAdjointPoints_cuda(ccs_Batch *batch);
/* The adjoint of a fitting loss's gradient direction, fused: gradCagePoints =
 * S^T (P - T), P = the refined points the last ccs_BatchRefinePoints_cuda
 * left, T = `target` (device, the points' layout).  The gradient of
 * mean ||P - T||^2 over the N points is 2/N times this.  The finest level of
 * every cage of depth >= 3 is read as P - T inside the first adjoint step;
 * the other levels are set to P - T in the gradPoints buffer first.  No
 * counterpart in the reference (which has no adjoint). */
int ccs_BatchAdjointDistance_cuda(ccs_Batch *batch, const float *target);
int ccs_BatchGetArrays_cuda(ccs_Batch *batch, ccs_BatchArrays *out);
int ccs_BatchCageInfo_cuda(const ccs_Batch *batch, int32_t cage, ccs_BatchCageInfo *out);
int ccs_BatchSetStream_cuda(ccs_Batch *batch, void *stream);
/* Persistent grid size: resident blocks per SM (0 = all that fit). */
int ccs_BatchSetSchedule_cuda(ccs_Batch *batch, int32_t blocksPerSM);
/* Launch schedule: 0 = one cooperative launch per depth with grid barriers
 * between its sections (default); 1 = one launch per section, each kernel
 * with its own register budget. */
int ccs_BatchSetLaunchMode_cuda(ccs_Batch *batch, int32_t split);
/* Waits for the batch's stream; CCS_ERR_TIMEOUT if a grid barrier gave up. */
int ccs_BatchSynchronize_cuda(ccs_Batch *batch);
/* Copies one cage's hierarchy into the host arrays of a cc_Subd made for
 * the same cage and depth (e.g. by the reference's ccs_Create). */
int ccs_BatchDownload_cuda(ccs_Batch *batch, int32_t cage, cc_Subd *subd);
/* Self-test of the bounded grid-barrier wait the batched kernels use: runs a
 * one-block barrier that waits for an arrival that never comes.  Returns
 * CCS_ERR_TIMEOUT when the wait gave up and reported as designed (the
 * expected result; the CUDA context stays usable), CCS_OK if it did not. */
int ccs_BarrierTimeoutSelfTest_cuda(void);

/* ---------------------------------------------------------------------- */
/* Counts (int64, with the int32 overflow check the library applies)       */
/* ---------------------------------------------------------------------- */
typedef struct {
    int64_t H, F, E, V, C;            /* counts at one depth                */
    int64_t cumH, cumC, cumV;         /* offset of this depth's arrays      */
} ccs_LevelCounts;
/* Level counts of depth 0..maxDepth (maxDepth+1 entries).  Returns
 * CCS_ERR_OVERFLOW when a count the reference stores in int32 would
 * overflow at that depth. */
int ccs_LevelCounts_cuda(const cc_Mesh *cage, int32_t maxDepth, ccs_LevelCounts *out);
/* Largest depth whose counts all fit the reference's int32 arithmetic. */
int32_t ccs_MaxSupportedDepth_cuda(const cc_Mesh *cage);

/* ---------------------------------------------------------------------- */
/* Kernel timing (profiling aid)                                           */
/* ---------------------------------------------------------------------- */
typedef struct {
    int32_t kernel;           /* CCS_K_* identifier                          */
    int32_t level;            /* parent depth the launch refines             */
    float ms;                 /* device time between CUDA events             */
    int64_t units;            /* parent halfedges / creases processed        */
} ccs_KernelTime;
enum {
    CCS_K_TOPOLOGY = 0, CCS_K_CREASES = 1, CCS_K_FACE_POINTS = 2, CCS_K_EDGE_POINTS = 3,
    CCS_K_VERTEX_POINTS = 4, CCS_K_CLEAR = 5, CCS_K_LEVEL_FUSED = 6, CCS_K_ADJOINT = 7,
    CCS_K_UVS = 8, CCS_K_LEVEL_POINTS = 9, CCS_K_OLD_VERTICES = 10, CCS_K_RING_STATS = 11,
    CCS_K_ADJ_EDGES = 12, CCS_K_ADJ_FACES = 13, CCS_K_ADJ_VERTICES = 14, CCS_K_EXACT_POINTS = 15,
    CCS_K_STEP = 16 /* a whole refinement step d -> d+1, on the subd's stream */,
    CCS_K_LEVEL_STEP = 17 /* depth >= 2: topology, creases and all points in one launch */,
    CCS_K_LEVEL_STEP_POINTS = 18 /* depth >= 2: all points of a step in one launch */,
    CCS_K_ADJ_STEP = 19 /* adjoint of a depth >= 2 step in one launch */,
    CCS_K_CREASE_STATS = 20 /* crease half of a level's ring statistics (ring_stats = the shape half) */,
    CCS_K_CAGE_SIDE = 21 /* cage topology, cage creases and every level's shape statistics in one launch */,
    CCS_K_CAGE_MAP = 22 /* the cage step's points as one sparse linear map (default pass) */,
    CCS_K_ADJ_CAGE_MAP = 23 /* the adjoint's cage level: the transposed map */,
    CCS_K_COUNT = 24
};
/* When enabled, every launch of the subd is bracketed by CUDA events.  A
 * refinement operation then replays a CUDA graph of its own whose event
 * record nodes time each launch as the graph runs it (the call waits for the
 * stream after each replay); with CCS_FLAG_NO_GRAPH, or while the caller
 * captures the stream, and for the adjoint entry points, the launches are
 * direct and the events are recorded on the stream. */
int ccs_SetProfiling_cuda(cc_Subd *subd, int enable);
/* Copies up to `cap` records of the launches since the last call (waits for
 * the stream); returns the number of records, or a negative status. */
int ccs_ReadProfile_cuda(cc_Subd *subd, ccs_KernelTime *out, int cap);
const char *ccs_KernelName_cuda(int kernel);

/* ---------------------------------------------------------------------- */
/* Errors                                                                  */
/* ---------------------------------------------------------------------- */
int ccs_LastError_cuda(void);                 /* last status of this thread */
const char *ccs_ErrorString_cuda(int status);
const char *ccs_Version_cuda(void);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* CCS_CUDA_H */
