/* ccs_cuda_compat.h -- source compatibility with CatmullClark.h's subd calls.
 *
 * Include it after CatmullClark.h (when that header is used at all): from
 * there on the reference's subd calls keep their names, argument lists and
 * void results (CatmullClark.h:145-146, :197-212) and run on the GPU.  Each
 * refinement call runs its ccs_*_cuda twin and then ccs_Download_cuda, which
 * copies the results into subd->halfedges / creases / vertexPoints and waits,
 * so code that reads them afterwards -- the accessors of CatmullClark.h:986-1395,
 * ExportToObj of examples/subd_cpu.c -- runs unchanged, and so does code that
 * takes the calls' addresses (Bench(&ccs_Refine_Scatter, subd) in
 * examples/subd_cpu.c).  A failing call leaves its status in
 * ccs_LastError_cuda(); nothing aborts.
 *
 * The cage stays the caller's: ccm_Load / ccm_Release are not renamed
 * (ccs_LoadCage_cuda / ccs_ReleaseCage_cuda load one into page-locked memory
 * instead).  A subd made by ccs_Create here is released by ccs_Release here.
 */
#ifndef CCS_CUDA_COMPAT_H
#define CCS_CUDA_COMPAT_H

#include "ccs_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* a refinement call's status, then the results to the host arrays */
static inline void ccs_compat_finish_(cc_Subd *subd, int status)
{
    if (status == CCS_OK)
        ccs_Download_cuda(subd);
}

/* ccs_Create's flags (CCS_FLAG_*), chosen when the program is compiled, as
 * the reference's own variants are (CC_DISABLE_UV): 0 by default; e.g.
 * -DCCS_COMPAT_FLAGS=CCS_FLAG_DETERMINISTIC sums every point in the
 * reference's one-thread order, bit for bit. */
#ifndef CCS_COMPAT_FLAGS
#define CCS_COMPAT_FLAGS 0u
#endif

static inline cc_Subd *ccs_compat_Create(const cc_Mesh *cage, int32_t maxDepth)
{
    cc_Subd *subd = NULL;
    return ccs_CreateEx_cuda(cage, maxDepth, (uint32_t)(CCS_COMPAT_FLAGS), &subd) == CCS_OK ? subd : NULL;
}
static inline void ccs_compat_Release(cc_Subd *subd)
{ ccs_Release_cuda(subd); }

static inline void ccs_compat_Refine_Scatter(cc_Subd *subd)
{ ccs_compat_finish_(subd, ccs_Refine_Scatter_cuda(subd)); }
static inline void ccs_compat_Refine_Gather(cc_Subd *subd)
{ ccs_compat_finish_(subd, ccs_Refine_Gather_cuda(subd)); }
static inline void ccs_compat_RefineVertexPoints_Scatter(cc_Subd *subd)
{ ccs_compat_finish_(subd, ccs_RefineVertexPoints_Scatter_cuda(subd)); }
static inline void ccs_compat_RefineVertexPoints_Gather(cc_Subd *subd)
{ ccs_compat_finish_(subd, ccs_RefineVertexPoints_Gather_cuda(subd)); }
static inline void ccs_compat_RefineHalfedges(cc_Subd *subd)
{ ccs_compat_finish_(subd, ccs_RefineHalfedges_cuda(subd)); }
static inline void ccs_compat_RefineCreases(cc_Subd *subd)
{ ccs_compat_finish_(subd, ccs_RefineCreases_cuda(subd)); }
static inline void ccs_compat_RefineVertexUvs(cc_Subd *subd)
{ ccs_compat_finish_(subd, ccs_RefineVertexUvs_cuda(subd)); }
static inline void ccs_compat_Refine_NoCreases_Scatter(cc_Subd *subd)
{ ccs_compat_finish_(subd, ccs_Refine_NoCreases_Scatter_cuda(subd)); }
static inline void ccs_compat_Refine_NoCreases_Gather(cc_Subd *subd)
{ ccs_compat_finish_(subd, ccs_Refine_NoCreases_Gather_cuda(subd)); }
static inline void ccs_compat_RefineVertexPoints_NoCreases_Scatter(cc_Subd *subd)
{ ccs_compat_finish_(subd, ccs_RefineVertexPoints_NoCreases_Scatter_cuda(subd)); }
static inline void ccs_compat_RefineVertexPoints_NoCreases_Gather(cc_Subd *subd)
{ ccs_compat_finish_(subd, ccs_RefineVertexPoints_NoCreases_Gather_cuda(subd)); }

#ifdef __cplusplus
}
#endif

#define ccs_Create                              ccs_compat_Create
#define ccs_Release                             ccs_compat_Release
#define ccs_Refine_Scatter                      ccs_compat_Refine_Scatter
#define ccs_Refine_Gather                       ccs_compat_Refine_Gather
#define ccs_RefineVertexPoints_Scatter          ccs_compat_RefineVertexPoints_Scatter
#define ccs_RefineVertexPoints_Gather           ccs_compat_RefineVertexPoints_Gather
#define ccs_RefineHalfedges                     ccs_compat_RefineHalfedges
#define ccs_RefineCreases                       ccs_compat_RefineCreases
#define ccs_RefineVertexUvs                     ccs_compat_RefineVertexUvs
#define ccs_Refine_NoCreases_Scatter            ccs_compat_Refine_NoCreases_Scatter
#define ccs_Refine_NoCreases_Gather             ccs_compat_Refine_NoCreases_Gather
#define ccs_RefineVertexPoints_NoCreases_Scatter ccs_compat_RefineVertexPoints_NoCreases_Scatter
#define ccs_RefineVertexPoints_NoCreases_Gather  ccs_compat_RefineVertexPoints_NoCreases_Gather

#endif /* CCS_CUDA_COMPAT_H */
