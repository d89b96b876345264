// ccs_ccm.cu -- `.ccm` cage files (ccm_Load / ccm_Save / ccm_Release of
// CatmullClark.h:3085-3269) read into one page-locked host block.
//
// File layout (the reference's x86-64 build, little-endian): a 32-byte
// header {int64 magic "cc_Mesh1", int32 vertexCount, uvCount, halfedgeCount,
// edgeCount, faceCount, 4 bytes of struct padding} (:3092-3139), then the
// vertex->halfedge, edge->halfedge and face->halfedge maps, the vertex
// points, the uvs, one crease per edge and the halfedges (:3162-3179).
//
// The loader puts a small block header, the cc_Mesh struct and all seven
// arrays in ONE allocation, pinned with cudaHostAlloc when the CUDA runtime
// can (plain malloc otherwise), so that ccs_Create_cuda's uploads are DMA
// copies straight out of the file's buffer with no staging copy.  Each array
// starts on a 64-byte boundary.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "ccs_host.h"

namespace ccs {

static constexpr uint64_t kBlockMagic = 0x6b636f6c426d6363ull;  // "ccmBlock"
static constexpr int64_t kAlign = 64;

struct CageBlock {
    uint64_t magic;
    int32_t pinned;     // 1: cudaHostAlloc, 0: malloc
    int32_t pad;
    int64_t bytes;
};

struct FileHeader {
    char magic[8];
    int32_t V, U, H, E, F;
    int32_t pad;
};
static_assert(sizeof(FileHeader) == 32, "ccm header is 32 bytes");
static_assert(sizeof(cc_Halfedge) == 28 && sizeof(cc_Crease) == 12, "record sizes of CatmullClark.h");

static const char kFileMagic[8] = {'c', 'c', '_', 'M', 'e', 's', 'h', '1'};

static int64_t up(int64_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// byte sizes of the seven arrays in file order
static void array_bytes(const FileHeader& h, int64_t out[7]) {
    out[0] = 4ll * h.V;
    out[1] = 4ll * h.E;
    out[2] = 4ll * h.F;
    out[3] = 12ll * h.V;
    out[4] = 8ll * h.U;
    out[5] = 12ll * h.E;
    out[6] = 28ll * h.H;
}

static CageBlock* block_of(cc_Mesh* m) {
    if (!m) return nullptr;
    CageBlock* b = reinterpret_cast<CageBlock*>(reinterpret_cast<char*>(m) - up(sizeof(CageBlock)));
    return b->magic == kBlockMagic ? b : nullptr;
}

static void free_block(CageBlock* b) {
    b->magic = 0;
    if (b->pinned) cudaFreeHost(b);
    else free(b);
}

// One block for a cage of these counts: the cc_Mesh with its counts set and
// its array pointers into the block (uvs NULL when U = 0).
cc_Mesh* alloc_cage_block(int32_t V, int32_t U, int32_t H, int32_t E, int32_t F) {
    FileHeader h;
    h.V = V; h.U = U; h.H = H; h.E = E; h.F = F;
    int64_t sz[7];
    array_bytes(h, sz);
    int64_t total = up(sizeof(CageBlock)) + up(sizeof(cc_Mesh));
    for (int i = 0; i < 7; ++i) total += up(sz[i]);
    char* base = nullptr;
    int pinned = 0;
    if (cudaHostAlloc(reinterpret_cast<void**>(&base), (size_t)total, cudaHostAllocDefault) == cudaSuccess) {
        pinned = 1;
    } else {
        cudaGetLastError();  // clear the failed call's status
        base = static_cast<char*>(malloc((size_t)total));
    }
    if (!base) return nullptr;
    CageBlock* b = reinterpret_cast<CageBlock*>(base);
    b->magic = kBlockMagic;
    b->pinned = pinned;
    b->pad = 0;
    b->bytes = total;
    cc_Mesh* m = reinterpret_cast<cc_Mesh*>(base + up(sizeof(CageBlock)));
    char* p = reinterpret_cast<char*>(m) + up(sizeof(cc_Mesh));
    char* arr[7];
    for (int i = 0; i < 7; ++i) {
        arr[i] = p;
        p += up(sz[i]);
    }
    m->vertexCount = V;
    m->uvCount = U;
    m->halfedgeCount = H;
    m->edgeCount = E;
    m->faceCount = F;
    m->vertexToHalfedgeIDs = reinterpret_cast<int32_t*>(arr[0]);
    m->edgeToHalfedgeIDs = reinterpret_cast<int32_t*>(arr[1]);
    m->faceToHalfedgeIDs = reinterpret_cast<int32_t*>(arr[2]);
    m->vertexPoints = reinterpret_cast<cc_VertexPoint*>(arr[3]);
    m->uvs = U > 0 ? reinterpret_cast<cc_VertexUv*>(arr[4]) : nullptr;
    m->creases = reinterpret_cast<cc_Crease*>(arr[5]);
    m->halfedges = reinterpret_cast<cc_Halfedge*>(arr[6]);
    return m;
}

void free_cage_block(cc_Mesh* m) {
    CageBlock* b = block_of(m);
    if (b) free_block(b);
}

}  // namespace ccs

using namespace ccs;

extern "C" {

cc_Mesh* ccs_LoadCage_cuda(const char* path) {
    set_last_error(CCS_ERR_ARG);
    if (!path) return nullptr;
    FILE* f = fopen(path, "rb");
    if (!f) return nullptr;
    FileHeader h;
    if (fread(&h, sizeof h, 1, f) != 1 || memcmp(h.magic, kFileMagic, 8) != 0 ||
        h.V < 0 || h.U < 0 || h.H < 0 || h.E < 0 || h.F < 0) {
        fclose(f);
        return nullptr;
    }
    cc_Mesh* m = alloc_cage_block(h.V, h.U, h.H, h.E, h.F);
    if (!m) {
        fclose(f);
        set_last_error(CCS_ERR_ALLOC);
        return nullptr;
    }
    // file order: v2h, e2h, f2h, points, uvs, creases, halfedges
    void* dst[7] = {m->vertexToHalfedgeIDs, m->edgeToHalfedgeIDs, m->faceToHalfedgeIDs, m->vertexPoints,
                    m->uvs, m->creases, m->halfedges};
    int64_t sz[7];
    array_bytes(h, sz);
    for (int i = 0; i < 7; ++i) {
        if (sz[i] > 0 && fread(dst[i], 1, (size_t)sz[i], f) != (size_t)sz[i]) {
            fclose(f);
            free_cage_block(m);
            return nullptr;
        }
    }
    fclose(f);
    set_last_error(CCS_OK);
    return m;
}

void ccs_ReleaseCage_cuda(cc_Mesh* cage) { free_cage_block(cage); }

int ccs_SaveCage_cuda(const cc_Mesh* m, const char* path) {
    if (!m || !path || m->vertexCount < 0 || m->uvCount < 0 || m->halfedgeCount < 0 || m->edgeCount < 0 ||
        m->faceCount < 0)
        return CCS_ERR_ARG;
    FileHeader h;
    memcpy(h.magic, kFileMagic, 8);
    h.V = m->vertexCount; h.U = m->uvCount; h.H = m->halfedgeCount; h.E = m->edgeCount; h.F = m->faceCount;
    h.pad = 0;
    int64_t sz[7];
    array_bytes(h, sz);
    const void* src[7] = {m->vertexToHalfedgeIDs, m->edgeToHalfedgeIDs, m->faceToHalfedgeIDs, m->vertexPoints,
                          m->uvs, m->creases, m->halfedges};
    for (int i = 0; i < 7; ++i)
        if (sz[i] > 0 && !src[i]) return CCS_ERR_ARG;
    FILE* f = fopen(path, "wb");
    if (!f) return CCS_ERR_ARG;
    bool ok = fwrite(&h, sizeof h, 1, f) == 1;
    for (int i = 0; ok && i < 7; ++i)
        ok = sz[i] == 0 || fwrite(src[i], 1, (size_t)sz[i], f) == (size_t)sz[i];
    ok = (fclose(f) == 0) && ok;
    return ok ? CCS_OK : CCS_ERR_ARG;
}

}  // extern "C"
