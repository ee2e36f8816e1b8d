// Restart files in the reference's record format (SRC/save_raw.F90:37-69,
// SRC/restore_raw.F90:35-61) for library-owned lattices.
//
// A restart file is a Fortran sequential unformatted file of 20 records: the
// time step (a 4-byte integer), then populations 01..19, each over the full
// halo box i = 0..l+1, j = 0..m+1, k = 0..n+1 with i fastest.  Each record
// is framed by 4-byte length markers (the gfortran / nvfortran default).  A
// record longer than 2147483639 bytes is split into subrecords the gfortran
// way: the leading marker of a subrecord that another one follows is
// negative, and so is the trailing marker of a subrecord that continues an
// earlier one.
//
// Records are streamed one population at a time through a device staging
// buffer, so a save or a restore needs one population's worth of extra device
// and host memory.  Values are either the stored elements as they are
// (file_bytes 0: for the 16-bit kinds, the scaled 16-bit patterns), or
// converted on the device to real*4 / real*8 (16-bit kinds unscaled), which
// is what a reference build of that precision reads.  A restore infers the
// file's element size from its record lengths: 2-byte records go as they are
// into a 16-bit lattice, and are read as IEEE half values into a 4- or 8-byte
// one (the reference's HALF storage).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "bgk_internal.h"
#include "d3q19.cuh"
#include "lattice_internal.h"

using namespace bgk;

namespace {

long long g_max_subrecord = 2147483639LL;   // gfortran's limit for 4-byte markers

// element conversions: physical value <-> storage element (scale applies to
// the 16-bit kinds)
template <class T> struct Elem;
template <> struct Elem<double> {
    static __device__ double to_d(double v, float) { return v; }
    static __device__ double from_d(double v, float) { return v; }
};
template <> struct Elem<float> {
    static __device__ double to_d(float v, float) { return (double)v; }
    static __device__ float from_d(double v, float) { return __double2float_rn(v); }
};
template <> struct Elem<__half> {
    static __device__ double to_d(__half v, float inv) { return (double)__fmul_rn(__half2float(v), inv); }
    static __device__ __half from_d(double v, float scl) { return __float2half_rn(__fmul_rn(__double2float_rn(v), scl)); }
};
template <> struct Elem<__nv_bfloat16> {
    static __device__ double to_d(__nv_bfloat16 v, float inv) { return (double)__fmul_rn(__bfloat162float(v), inv); }
    static __device__ __nv_bfloat16 from_d(double v, float scl) {
        return __float2bfloat16_rn(__fmul_rn(__double2float_rn(v), scl));
    }
};

// padded plane (element (0,0,0) at `plane`, pitches nx, nx*ny) -> dense box
template <class S, class F>
__global__ void pack_box_kernel(const S* __restrict__ plane, F* __restrict__ box, long long nx, long long nxy,
                                int ni, int nj, long long npts, float s_inv, float f_scale) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= npts) return;
    const long long i = t % ni, j = (t / ni) % nj, k = t / ((long long)ni * nj);
    box[t] = Elem<F>::from_d(Elem<S>::to_d(plane[i + nx * j + nxy * k], s_inv), f_scale);
}

// dense box -> padded plane
template <class F, class S>
__global__ void unpack_box_kernel(const F* __restrict__ box, S* __restrict__ plane, long long nx, long long nxy,
                                  int ni, int nj, long long npts, float f_inv, float s_scale) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= npts) return;
    const long long i = t % ni, j = (t / ni) % nj, k = t / ((long long)ni * nj);
    plane[i + nx * j + nxy * k] = Elem<S>::from_d(Elem<F>::to_d(box[t], f_inv), s_scale);
}

struct Shape {
    int ni, nj, nk;
    long long npts, nx, nxy;
};

Shape shape_of(const bgk_lattice* L) {
    Shape s;
    s.ni = L->desc.l + 2; s.nj = L->desc.m + 2; s.nk = L->desc.n + 2;
    s.npts = (long long)s.ni * s.nj * s.nk;
    s.nx = L->nx; s.nxy = L->nx * L->ny;
    return s;
}

bool is16(int kind) { return kind == K_F16 || kind == K_BF16; }
float storage_scale(const bgk_lattice* L) { return is16(L->desc.kind) ? L->desc.scale : 1.0f; }

template <class S, class F>
int launch_pack(const void* plane, void* box, const Shape& s, float s_scale, cudaStream_t st) {
    const unsigned grid = (unsigned)((s.npts + 255) / 256);
    pack_box_kernel<S, F><<<grid, 256, 0, st>>>((const S*)plane, (F*)box, s.nx, s.nxy, s.ni, s.nj, s.npts,
                                                1.0f / s_scale, 1.0f);
    return check_launch("pack_box_kernel");
}

template <class F, class S>
int launch_unpack(const void* box, void* plane, const Shape& s, float s_scale, cudaStream_t st) {
    const unsigned grid = (unsigned)((s.npts + 255) / 256);
    unpack_box_kernel<F, S><<<grid, 256, 0, st>>>((const F*)box, (S*)plane, s.nx, s.nxy, s.ni, s.nj, s.npts,
                                                  1.0f, s_scale);
    return check_launch("unpack_box_kernel");
}

// storage kind S of the lattice -> file element F (fb = 2: IEEE half, 4, 8)
template <class F>
int pack_any(int kind, const void* plane, void* box, const Shape& s, float scl, cudaStream_t st) {
    switch (kind) {
        case K_F64: return launch_pack<double, F>(plane, box, s, 1.0f, st);
        case K_F32: case K_F32_F64: return launch_pack<float, F>(plane, box, s, 1.0f, st);
        case K_F16: return launch_pack<__half, F>(plane, box, s, scl, st);
        default: return launch_pack<__nv_bfloat16, F>(plane, box, s, scl, st);
    }
}

template <class F>
int unpack_any(int kind, const void* box, void* plane, const Shape& s, float scl, cudaStream_t st) {
    switch (kind) {
        case K_F64: return launch_unpack<F, double>(box, plane, s, 1.0f, st);
        case K_F32: case K_F32_F64: return launch_unpack<F, float>(box, plane, s, 1.0f, st);
        case K_F16: return launch_unpack<F, __half>(box, plane, s, scl, st);
        default: return launch_unpack<F, __nv_bfloat16>(box, plane, s, scl, st);
    }
}

struct FileCloser {
    void operator()(FILE* f) const { if (f) std::fclose(f); }
};
using File = std::unique_ptr<FILE, FileCloser>;

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

bool put_marker(FILE* f, long long v) {
    const int32_t m = (int32_t)v;
    return std::fwrite(&m, 4, 1, f) == 1;
}

// one logical record, split into subrecords when longer than g_max_subrecord
bool write_record(FILE* f, const char* data, long long bytes) {
    long long off = 0;
    bool first = true;
    do {
        const long long len = std::min(bytes - off, g_max_subrecord);
        const bool more = off + len < bytes;
        if (!put_marker(f, more ? -len : len)) return false;
        if (len && std::fwrite(data + off, 1, (size_t)len, f) != (size_t)len) return false;
        if (!put_marker(f, first ? len : -len)) return false;
        off += len;
        first = false;
    } while (off < bytes);
    return true;
}

// length of the next logical record (all subrecords), file position unchanged
bool record_length(FILE* f, long long* bytes) {
    const long pos = std::ftell(f);
    long long total = 0;
    for (;;) {
        int32_t head, tail;
        if (std::fread(&head, 4, 1, f) != 1) return false;
        const long long len = head < 0 ? -(long long)head : head;
        if (std::fseek(f, (long)len, SEEK_CUR) != 0) return false;
        if (std::fread(&tail, 4, 1, f) != 1) return false;
        if ((tail < 0 ? -(long long)tail : tail) != len) return false;
        total += len;
        if (head >= 0) break;
    }
    *bytes = total;
    return std::fseek(f, pos, SEEK_SET) == 0;
}

bool skip_record(FILE* f) {
    for (;;) {
        int32_t head;
        if (std::fread(&head, 4, 1, f) != 1) return false;
        const long long len = head < 0 ? -(long long)head : head;
        if (std::fseek(f, (long)len + 4, SEEK_CUR) != 0) return false;
        if (head >= 0) return true;
    }
}

bool read_record(FILE* f, char* data, long long bytes) {
    long long off = 0;
    for (;;) {
        int32_t head, tail;
        if (std::fread(&head, 4, 1, f) != 1) return false;
        const long long len = head < 0 ? -(long long)head : head;
        if (off + len > bytes) return false;
        if (len && std::fread(data + off, 1, (size_t)len, f) != (size_t)len) return false;
        if (std::fread(&tail, 4, 1, f) != 1) return false;
        off += len;
        if (head >= 0) break;
    }
    return off == bytes;
}

}  // namespace

extern "C" {

long long bgk_io_set_subrecord_limit(long long bytes) {
    const long long prev = g_max_subrecord;
    if (bytes >= 4 && bytes <= 2147483639LL) g_max_subrecord = bytes;
    return prev;
}

int bgk_lattice_save(const bgk_lattice* L, const char* path, int itime, int file_bytes, void* stream) {
    if (!L || !path) return set_error(BGK_ERR_ARG, "null argument");
    if (file_bytes != 0 && file_bytes != 4 && file_bytes != 8)
        return set_error(BGK_ERR_ARG, "file_bytes must be 0 (as stored), 4 or 8, not %d", file_bytes);
    if (L->desc.pattern == BGK_PATTERN_AA && (L->steps % 2) != 0)
        return set_error(BGK_ERR_STATE, "AA lattice after an odd number of steps holds no observable state");
    cudaStream_t st = (cudaStream_t)stream;
    const Shape s = shape_of(L);
    const int fb = file_bytes ? file_bytes : L->es;
    const long long rec = s.npts * fb;
    std::vector<char> host((size_t)rec);
    DevBuf box;
    const bool convert = file_bytes != 0 && file_bytes != L->es;
    if (convert) {
        cudaError_t e = cudaMalloc(&box.p, (size_t)rec);
        if (e != cudaSuccess) return set_error(BGK_ERR_NOMEM, "save staging: %s", cudaGetErrorString(e));
    }
    File f(std::fopen(path, "wb"));
    if (!f) return set_error(BGK_ERR_ARG, "cannot open %s for writing", path);
    const int32_t it = itime;
    if (!write_record(f.get(), (const char*)&it, 4)) return set_error(BGK_ERR_ARG, "write failed: %s", path);
    void* src[19];
    bgk_lat::observable(L, src);
    const float scl = storage_scale(L);
    for (int d = 0; d < 19; ++d) {
        cudaError_t e;
        if (convert) {
            const int rc = fb == 4 ? pack_any<float>(L->desc.kind, src[d], box.p, s, scl, st)
                                   : pack_any<double>(L->desc.kind, src[d], box.p, s, scl, st);
            if (rc) return rc;
            e = cudaMemcpyAsync(host.data(), box.p, (size_t)rec, cudaMemcpyDeviceToHost, st);
        } else {
            const size_t row = (size_t)s.ni * L->es;
            e = cudaMemcpy2DAsync(host.data(), row, src[d], (size_t)L->nx * L->es, row, (size_t)s.nj * s.nk,
                                  cudaMemcpyDeviceToHost, st);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "save copy: %s", cudaGetErrorString(e));
        if (!write_record(f.get(), host.data(), rec)) return set_error(BGK_ERR_ARG, "write failed: %s", path);
    }
    if (std::fflush(f.get()) != 0) return set_error(BGK_ERR_ARG, "write failed: %s", path);
    return BGK_OK;
}

int bgk_lattice_restore(bgk_lattice* L, const char* path, int* itime, void* stream) {
    if (!L || !path) return set_error(BGK_ERR_ARG, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const Shape s = shape_of(L);
    File f(std::fopen(path, "rb"));
    if (!f) return set_error(BGK_ERR_ARG, "cannot open %s", path);
    long long len = 0;
    int32_t it = 0;
    if (!record_length(f.get(), &len) || len != 4 || !read_record(f.get(), (char*)&it, 4))
        return set_error(BGK_ERR_ARG, "%s: first record is not a 4-byte time step", path);
    if (!record_length(f.get(), &len) || len % s.npts != 0)
        return set_error(BGK_ERR_ARG, "%s: population record of %lld bytes does not hold %dx%dx%d values", path,
                         len, s.ni, s.nj, s.nk);
    const int fb = (int)(len / s.npts);
    if (fb != 2 && fb != 4 && fb != 8)
        return set_error(BGK_ERR_ARG, "%s: %d bytes per value", path, fb);
    const bool raw = fb == L->es;
    std::vector<char> host((size_t)len);
    DevBuf box;
    if (!raw) {
        cudaError_t e = cudaMalloc(&box.p, (size_t)len);
        if (e != cudaSuccess) return set_error(BGK_ERR_NOMEM, "restore staging: %s", cudaGetErrorString(e));
    }
    // check every record's framing before touching the lattice, so a short or
    // damaged file leaves the lattice as it was
    const long first = std::ftell(f.get());
    for (int d = 0; d < 19; ++d) {
        long long l2 = 0;
        if (!record_length(f.get(), &l2) || l2 != len || !skip_record(f.get()))
            return set_error(BGK_ERR_ARG, "%s: record %d is missing or has %lld bytes, expected %lld", path, d + 2,
                             l2, len);
    }
    std::fseek(f.get(), first, SEEK_SET);
    void* dst[19];
    bgk_lat::begin_load(L, dst);
    const float scl = storage_scale(L);
    for (int d = 0; d < 19; ++d) {
        if (!read_record(f.get(), host.data(), len)) return set_error(BGK_ERR_ARG, "%s: short record %d", path, d + 2);
        cudaError_t e;
        if (raw) {
            const size_t row = (size_t)s.ni * L->es;
            e = cudaMemcpy2DAsync(dst[d], (size_t)L->nx * L->es, host.data(), row, row, (size_t)s.nj * s.nk,
                                  cudaMemcpyHostToDevice, st);
        } else {
            e = cudaMemcpyAsync(box.p, host.data(), (size_t)len, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) {
                const int rc = fb == 2 ? unpack_any<__half>(L->desc.kind, box.p, dst[d], s, scl, st)
                             : fb == 4 ? unpack_any<float>(L->desc.kind, box.p, dst[d], s, scl, st)
                                       : unpack_any<double>(L->desc.kind, box.p, dst[d], s, scl, st);
                if (rc) return rc;
            }
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return set_error(BGK_ERR_CUDA, "restore copy: %s", cudaGetErrorString(e));
    }
    if (itime) *itime = it;
    return bgk_lat::end_load(L, st);
}

}  // extern "C"
