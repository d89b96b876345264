// ccs_export.cu -- OBJ export of one depth of a refined subd, formatted on
// the GPU.
//
// Writes the bytes the reference's ExportToObj writes (examples/subd_cpu.c:
// 22-115): "# Vertices", one "v %f %f %f" line per vertex point of the
// depth, then "vt %f %f" lines (the cage's texture points at depth 0; at
// depth >= 1 one per halfedge, its decoded uvID, CatmullClark.h:374-383 --
// none for 12-byte records, the CC_DISABLE_UV build), a blank line,
// "# Topology", and one "f" line per face ("%i/%i" corners: vertex + 1 and
// texture index + 1; at depth >= 1 the texture index of corner k of face f is
// the halfedge 4 f + k; "%i" corners for 12-byte records), then a blank line
// at depth >= 1.
//
// One thread per line: a first pass measures every line, a 64-bit exclusive
// scan gives each line its offset, a second pass writes it; the host inserts
// the fixed headers and streams the text to the file through a page-locked
// buffer.  printf's "%f" is reproduced exactly: a float is m * 2^e, its value
// times 10^6 is m * 10^6 / 2^-e (below 2^44 / 2^-e), rounded to the nearest
// integer with ties to even, as glibc rounds the exact binary value.
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "ccs_host.h"
#include "ccs_internal.cuh"
#include "ccs_scan.cuh"

namespace ccs {
namespace {

constexpr int kB = 256;

// Appends text at o + n (o == nullptr: counts only).
struct Emit {
    char* o;
    int64_t n;
    __device__ void c(char ch) {
        if (o) o[n] = ch;
        ++n;
    }
    __device__ void s(const char* str) {
        while (*str) c(*str++);
    }
    __device__ void u64(uint64_t v) {
        char t[20];
        int k = 0;
        do { t[k++] = (char)('0' + v % 10); v /= 10; } while (v);
        while (k) c(t[--k]);
    }
    __device__ void u128(unsigned __int128 v) {
        char t[40];
        int k = 0;
        do { t[k++] = (char)('0' + (int)(v % 10)); v /= 10; } while (v);
        while (k) c(t[--k]);
    }
    __device__ void i32(int32_t v) {
        if (v < 0) {
            c('-');
            u64((uint64_t)(-(int64_t)v));
        } else {
            u64((uint64_t)v);
        }
    }
    // printf("%f", (double)x)
    __device__ void f6(float x) {
        const uint32_t b = __float_as_uint(x);
        const bool neg = (b >> 31) != 0;
        const uint32_t ex = (b >> 23) & 0xFFu, fr = b & 0x7FFFFFu;
        if (neg) c('-');
        if (ex == 0xFFu) {
            s(fr ? "nan" : "inf");
            return;
        }
        const uint64_t m = ex ? (fr | 0x800000u) : fr;
        const int e = ex ? (int)ex - 150 : -149;
        if (e >= 0) {
            if (e <= 39) u64(m << e);
            else u128((unsigned __int128)m << e);
            s(".000000");
            return;
        }
        const int k = -e;
        const uint64_t P = m * 1000000ull;           // below 2^44
        uint64_t q = 0;
        if (k < 64) {
            q = P >> k;
            const uint64_t r = P & ((1ull << k) - 1), half = 1ull << (k - 1);
            if (r > half || (r == half && (q & 1))) ++q;
        }
        u64(q / 1000000);
        c('.');
        const uint32_t f = (uint32_t)(q % 1000000);
        for (uint32_t d = 100000; d >= 1; d /= 10) c((char)('0' + (f / d) % 10));
    }
};

struct ObjArgs {
    int32_t depth, rw;
    int32_t V, T, F;                 // vertex, texture and face lines
    const float* pts;                // the depth's points
    const float* uvs;                // cage texture points (depth 0)
    const int32_t* he;               // depth >= 1: the depth's records; 0: cage records
    const int32_t* f2h;              // depth 0
};

__device__ void emit_line(const ObjArgs& a, int64_t i, Emit& e) {
    if (i < a.V) {
        const float* p = a.pts + 3 * i;
        e.s("v "); e.f6(p[0]); e.c(' '); e.f6(p[1]); e.c(' '); e.f6(p[2]); e.c('\n');
        return;
    }
    i -= a.V;
    if (i < a.T) {
        float u, v;
        if (a.depth == 0) {
            u = a.uvs[2 * i];
            v = a.uvs[2 * i + 1];
        } else {
            const uint32_t x = (uint32_t)a.he[(int64_t)a.rw * i + 3];
            u = __fdiv_rn((float)(x & 0xFFFFu), 65535.0f);
            v = __fdiv_rn((float)((x >> 16) & 0xFFFFu), 65535.0f);
        }
        e.s("vt "); e.f6(u); e.c(' '); e.f6(v); e.c('\n');
        return;
    }
    i -= a.T;                                         // face i
    if (a.depth == 0) {
        const int32_t h0 = a.f2h[i];
        const int32_t* r = a.he + (int64_t)CH_WORDS * h0;
        e.s("f "); e.i32(r[CH_VERT] + 1); e.c('/'); e.i32(r[CH_UV] + 1);
        int guard = 0;
        for (int32_t h = r[CH_NEXT]; h != h0 && guard < kWalkCap; h = a.he[(int64_t)CH_WORDS * h + CH_NEXT], ++guard) {
            const int32_t* q = a.he + (int64_t)CH_WORDS * h;
            e.c(' '); e.i32(q[CH_VERT] + 1); e.c('/'); e.i32(q[CH_UV] + 1);
        }
        e.c('\n');
        return;
    }
    e.c('f');
    for (int k = 0; k < 4; ++k) {
        const int64_t h = 4 * i + k;
        e.c(' ');
        e.i32(a.he[(int64_t)a.rw * h + 2] + 1);
        if (a.rw == 4) { e.c('/'); e.i32((int32_t)(h + 1)); }
    }
    e.c('\n');
}

__global__ void __launch_bounds__(kB) k_obj_len(ObjArgs a, int64_t L, int64_t* __restrict__ len) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L) return;
    Emit e{nullptr, 0};
    emit_line(a, i, e);
    len[i] = e.n;
}

__global__ void __launch_bounds__(kB) k_obj_write(ObjArgs a, int64_t L, const int64_t* __restrict__ off,
                                                  char* __restrict__ text) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L) return;
    Emit e{text + off[i], 0};
    emit_line(a, i, e);
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

int export_obj(const cc_Subd* subd, int32_t depth, const char* path) {
    SubdView sv;
    if (!path || !subd_view(subd, &sv) || depth < 0 || depth > sv.D) return CCS_ERR_ARG;
    if (depth > 0 && !sv.topo) return CCS_ERR_STATE;
    DeviceGuard g(sv.device);
    ObjArgs a;
    a.depth = depth;
    a.rw = sv.rw;
    if (depth == 0) {
        a.V = sv.cage->V; a.T = sv.cage->U; a.F = sv.cage->F;
        a.pts = sv.cage->pts; a.uvs = sv.cage->uvs; a.he = sv.cage->he; a.f2h = sv.cage->f2h;
    } else {
        const Level& lv = sv.lv[depth];
        a.V = lv.V; a.T = sv.rw == 4 ? lv.H : 0; a.F = lv.F;
        a.pts = sv.pts + 3 * lv.ptOff; a.uvs = nullptr; a.he = sv.he + (int64_t)sv.rw * lv.heOff; a.f2h = nullptr;
    }
    const int64_t L = (int64_t)a.V + a.T + a.F;
    const cudaStream_t s = sv.stream;
    DevBuf len, off, tiles, text;
    if (cudaMalloc(&len.p, sizeof(int64_t) * (size_t)L) != cudaSuccess ||
        cudaMalloc(&off.p, sizeof(int64_t) * ((size_t)L + 1)) != cudaSuccess ||
        cudaMalloc(&tiles.p, sizeof(int64_t) * (size_t)scan_tiles(L)) != cudaSuccess)
        return CCS_ERR_ALLOC;
    int64_t* dl = static_cast<int64_t*>(len.p);
    int64_t* doff = static_cast<int64_t*>(off.p);
    const unsigned nb = (unsigned)((L + kB - 1) / kB);
    k_obj_len<<<nb, kB, 0, s>>>(a, L, dl);
    if (exclusive_scan<int64_t>(dl, doff, L, static_cast<int64_t*>(tiles.p), doff + L, s) != cudaSuccess)
        return CCS_ERR_CUDA;
    int64_t total = 0, split = 0;
    if (cudaMemcpyAsync(&total, doff + L, sizeof(int64_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        (a.F > 0 && a.V + a.T < L &&
         cudaMemcpyAsync(&split, doff + a.V + a.T, sizeof(int64_t), cudaMemcpyDeviceToHost, s) != cudaSuccess) ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return CCS_ERR_CUDA;
    if (a.F == 0) split = total;
    if (cudaMalloc(&text.p, (size_t)(total > 0 ? total : 1)) != cudaSuccess) return CCS_ERR_ALLOC;
    k_obj_write<<<nb, kB, 0, s>>>(a, L, doff, static_cast<char*>(text.p));
    if (cudaGetLastError() != cudaSuccess) return CCS_ERR_CUDA;

    FILE* f = fopen(path, "wb");
    if (!f) return CCS_ERR_ARG;
    const size_t chunk = (size_t)64 << 20;
    char* stage = nullptr;
    if (cudaHostAlloc(reinterpret_cast<void**>(&stage), chunk, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        fclose(f);
        return CCS_ERR_ALLOC;
    }
    bool ok = true;
    auto put = [&](const char* str) { ok = ok && fwrite(str, 1, strlen(str), f) == strlen(str); };
    auto copy = [&](int64_t b, int64_t e) {
        for (int64_t p = b; ok && p < e; p += (int64_t)chunk) {
            const size_t n = (size_t)((e - p) < (int64_t)chunk ? (e - p) : (int64_t)chunk);
            ok = cudaMemcpyAsync(stage, static_cast<char*>(text.p) + p, n, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
                 cudaStreamSynchronize(s) == cudaSuccess && fwrite(stage, 1, n, f) == n;
        }
    };
    put("# Vertices\n");
    copy(0, split);
    put("\n# Topology\n");
    copy(split, total);
    if (depth > 0) put("\n");
    cudaFreeHost(stage);
    ok = (fclose(f) == 0) && ok;
    return ok ? CCS_OK : CCS_ERR_CUDA;
}

}  // namespace
}  // namespace ccs

extern "C" int ccs_ExportObj_cuda(const cc_Subd* subd, int32_t depth, const char* path) {
    return ccs::set_last_error(ccs::export_obj(subd, depth, path));
}
