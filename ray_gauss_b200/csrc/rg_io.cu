// Binary PLY vertex records -> FP32 columns on the device.
//
// The reference reads PLY files with numpy (scripts/ply.py:85-146: header, then np.fromfile of the
// vertex records as one structured array) and copies fields out column by column into torch tensors
// (classes/point_cloud.py:298-394, 396-495).  Here the host reads the record block once into pinned
// memory, copies it to the device in one transfer, and k_records_to_columns stages tiles of records
// in shared memory with coalesced loads and writes every requested field of every record to its
// destination column, converting the stored type (8- to 64-bit integers and floats, either byte
// order) to FP32.  A field may carry the affine map of the reference's colour initialisation,
// evaluated in double like numpy: ((v / div) + add) * mul_a * mul_b, then rounded to float once.
#include <cstdint>
#include <cstring>

#include "rg_common.cuh"

namespace {

constexpr int kIoThreads = 256;
constexpr int kIoSmem = 36 * 1024;     // record tile; the field descriptors take 10 KB beside it
// 10 KB of field descriptors in the kernel parameters (CUDA 12.1+ allows 32 KB on sm_70 and later):
// a trained scene's ~116 fields take one launch, so the records are staged once
constexpr int kFieldsPerLaunch = 160;

struct IoArgs {
    rg_record_field f[kFieldsPerLaunch];
    int n_fields;
    int record_bytes;
    int tile;                 // records per tile
    long long n;
    const unsigned char* rec;
};

__device__ __forceinline__ unsigned long long load_bytes(const unsigned char* p, int size, bool big) {
    unsigned long long v = 0;
    for (int b = 0; b < size; ++b) {
        const unsigned long long byte = p[b];
        v |= big ? byte << (8 * (size - 1 - b)) : byte << (8 * b);
    }
    return v;
}

__device__ double field_value(const unsigned char* p, int type, bool big) {
    switch (type) {
        case RG_FIELD_I8: return (double)(signed char)load_bytes(p, 1, big);
        case RG_FIELD_U8: return (double)(unsigned char)load_bytes(p, 1, big);
        case RG_FIELD_I16: return (double)(short)load_bytes(p, 2, big);
        case RG_FIELD_U16: return (double)(unsigned short)load_bytes(p, 2, big);
        case RG_FIELD_I32: return (double)(int)load_bytes(p, 4, big);
        case RG_FIELD_U32: return (double)(unsigned)load_bytes(p, 4, big);
        case RG_FIELD_F32: return (double)__uint_as_float((unsigned)load_bytes(p, 4, big));
        default: return __longlong_as_double((long long)load_bytes(p, 8, big));  // RG_FIELD_F64
    }
}

__global__ void __launch_bounds__(kIoThreads) k_records_to_columns(const IoArgs a) {
    extern __shared__ unsigned char tile[];
    // descriptors in shared memory: neighbouring lanes read different fields, which from the
    // kernel parameters would serialise on the constant cache
    __shared__ rg_record_field fs[kFieldsPerLaunch];
    for (int i = threadIdx.x; i < a.n_fields; i += kIoThreads) fs[i] = a.f[i];
    const long long r0 = (long long)blockIdx.x * a.tile;
    const int nr = (int)(r0 + a.tile <= a.n ? a.tile : a.n - r0);
    const long long bytes = (long long)nr * a.record_bytes;
    const unsigned char* src = a.rec + r0 * a.record_bytes;
    // stage the tile: 16-byte loads when the tile start and size allow, bytes otherwise
    if (((reinterpret_cast<uintptr_t>(src) | (uintptr_t)bytes) & 15) == 0) {
        const uint4* s4 = reinterpret_cast<const uint4*>(src);
        uint4* d4 = reinterpret_cast<uint4*>(tile);
        for (long long i = threadIdx.x; i < bytes / 16; i += kIoThreads) d4[i] = s4[i];
    } else {
        for (long long i = threadIdx.x; i < bytes; i += kIoThreads) tile[i] = src[i];
    }
    __syncthreads();
    // consecutive threads take consecutive fields of one record: the fields of a tensor row are
    // consecutive in the file (x y z, sh0r sh1r .., sx sy sz), so the stores coalesce
    for (int i = threadIdx.x; i < nr * a.n_fields; i += kIoThreads) {
        const int r = i / a.n_fields, fi = i - r * a.n_fields;
        const rg_record_field& f = fs[fi];
        const unsigned char* src_b = tile + (long long)r * a.record_bytes + f.offset;
        float out;
        if (f.type == RG_FIELD_F32 && !f.affine && ((uintptr_t)src_b & 3) == 0) {
            // float32 as stored: one aligned word (byte-swapped for big-endian files)
            unsigned u = *reinterpret_cast<const unsigned*>(src_b);
            if (f.big_endian) u = __byte_perm(u, 0, 0x0123);
            out = __uint_as_float(u);
        } else {
            double v = field_value(src_b, f.type, f.big_endian != 0);
            if (f.affine) v = ((v / f.div) + f.add) * f.mul_a * f.mul_b;
            out = (float)v;
        }
        f.dst[(r0 + r) * f.dst_stride] = out;
    }
}

int field_size(int type) {
    switch (type) {
        case RG_FIELD_I8: case RG_FIELD_U8: return 1;
        case RG_FIELD_I16: case RG_FIELD_U16: return 2;
        case RG_FIELD_I32: case RG_FIELD_U32: case RG_FIELD_F32: return 4;
        case RG_FIELD_F64: return 8;
        default: return 0;
    }
}

}  // namespace

extern "C" {

int rg_records_to_columns(const void* records, int64_t n, int32_t record_bytes, const rg_record_field* fields,
                          int32_t n_fields, void* stream) {
    if (n < 0 || record_bytes <= 0 || record_bytes > kIoSmem || n_fields < 0 ||
        n_fields > RG_RECORD_MAX_FIELDS || (n_fields && !fields))
        return RG_ERR_INVALID_ARG;
    for (int i = 0; i < n_fields; ++i) {
        const rg_record_field& f = fields[i];
        const int sz = field_size(f.type);
        if (!sz || f.offset < 0 || f.offset + sz > record_bytes || f.dst_stride <= 0 || (n > 0 && !f.dst))
            return RG_ERR_INVALID_ARG;
        if (f.affine && !(f.div != 0.0)) return RG_ERR_INVALID_ARG;
    }
    if (n == 0 || n_fields == 0) return RG_OK;
    if (!records) return RG_ERR_INVALID_ARG;
    IoArgs a;
    std::memset(&a, 0, sizeof(a));
    a.record_bytes = record_bytes;
    a.tile = kIoSmem / record_bytes;
    if (a.tile > 1024) a.tile = 1024;
    a.n = n;
    a.rec = static_cast<const unsigned char*>(records);
    const long long blocks = (n + a.tile - 1) / a.tile;
    const size_t smem = (size_t)a.tile * record_bytes;
    // fields in groups of kFieldsPerLaunch, each launch staging the records again
    for (int f0 = 0; f0 < n_fields; f0 += kFieldsPerLaunch) {
        a.n_fields = n_fields - f0 < kFieldsPerLaunch ? n_fields - f0 : kFieldsPerLaunch;
        std::memcpy(a.f, fields + f0, sizeof(rg_record_field) * a.n_fields);
        k_records_to_columns<<<(unsigned)blocks, kIoThreads, smem, reinterpret_cast<cudaStream_t>(stream)>>>(a);
        if (cudaGetLastError() != cudaSuccess) return RG_ERR_CUDA;
    }
    return RG_OK;
}

}  // extern "C"
