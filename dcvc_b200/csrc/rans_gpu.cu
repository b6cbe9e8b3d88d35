#include "rans_gpu.cuh"

#include "common.cuh"
#include "host_util.h"

#include <vector>

namespace dcvc {

namespace {

// The coder constants of rans_coder.cpp (rans.cpp:13-19 in the reference).
constexpr int kScaleBits = 16;
constexpr uint32_t kRansL = 1u << 23;
constexpr int kRenormShift = 23 - kScaleBits + 8;
constexpr uint32_t kBypassMax = 3;
constexpr uint32_t kBypassXMax = (1u << (kScaleBits - 2)) << kRenormShift;

struct EncJobs {
    RansGpuEncJob j[kRansGpuMaxJobs];
};
struct DecJobs {
    RansGpuDecJob j[kRansGpuMaxJobs];
};

__host__ __device__ inline void split(int n, int parts, int i, int* begin, int* end)
{
    const int s = n / parts;
    *begin = s * i;
    *end = (i < parts - 1) ? *begin + s : n;
}

__host__ __device__ inline int lane_cap(int n_y, int n_z, int ecp, int i)
{
    int b, e, bz, ez;
    split(n_y, ecp, i, &b, &e);
    split(n_z, ecp, i, &bz, &ez);
    return 4 * ((e - b) + (ez - bz)) + 16;
}

// One sub-stream's writer: bytes are produced back to front into [base, base + cap).
struct Writer {
    uint8_t* base;
    int pos;
    uint32_t x;
    bool overflow;
    bool zero_freq;  // a symbol with zero probability in its table (cannot be coded)

    __device__ void byte(uint32_t b)
    {
        if (pos == 0) {
            overflow = true;
            return;
        }
        base[--pos] = static_cast<uint8_t>(b);
    }
    __device__ void put(uint32_t start, uint32_t freq)
    {
        if (freq == 0) {
            zero_freq = true;
            return;
        }
        const uint32_t x_max = freq << kRenormShift;
        while (x >= x_max) {
            byte(x);
            x >>= 8;
        }
        x = ((x / freq) << kScaleBits) + (x % freq) + start;
    }
    __device__ void bits(uint32_t v)
    {
        while (x >= kBypassXMax) {
            byte(x);
            x >>= 8;
        }
        x = (x << 2) | v;
    }
    // Writer::symbol of rans_coder.cpp: symbol order 0, +1, -1, ...; values at or past the
    // table's max_value escape to 2-bit bypass digits (rans.cpp:144-181).
    __device__ void symbol(int32_t s, int32_t maxv, const uint32_t* enc)
    {
        int32_t v = (s < 0 ? -s : s) * 2 - (s > 0);
        if (v >= maxv) {
            const uint32_t raw = static_cast<uint32_t>(v - maxv);
            uint32_t bins[40];
            int nb = 0;
            int digits = 0;
            while (digits < 16 && (raw >> (digits * 2)) != 0) {
                ++digits;
            }
            int32_t cnt = digits;
            while (cnt >= static_cast<int32_t>(kBypassMax)) {
                bins[nb++] = kBypassMax;
                cnt -= kBypassMax;
            }
            bins[nb++] = static_cast<uint32_t>(cnt);
            for (int j = 0; j < digits; ++j) {
                bins[nb++] = (raw >> (2 * j)) & kBypassMax;
            }
            for (int j = nb - 1; j >= 0; --j) {
                bits(bins[j]);
            }
            v = maxv;
        }
        const uint32_t e = __ldg(enc + v);
        put(e & 0xffff, e >> 16);
    }
};

__device__ int shared_tail(const uint8_t* a, int na, const uint8_t* b, int nb)
{
    const int lim = min(min(na, nb), 8);
    int k = 0;
    for (int i = 0; i < lim; ++i) {
        if (a[na - 1 - i] != 0 || b[nb - 1 - i] != 0) {
            break;
        }
        ++k;
    }
    if (k == 0 && a[na - 1] == b[nb - 1]) {
        k = 1;
    }
    return k;
}

__device__ void put_i32(uint8_t* p, int32_t v)
{
    for (int k = 0; k < 4; ++k) {
        p[k] = static_cast<uint8_t>(static_cast<uint32_t>(v) >> (8 * k));
    }
}

__global__ void __launch_bounds__(32) rans_gpu_encode_kernel(RansGpuTables t, EncJobs jobs)
{
    griddep_launch_dependents();
    griddep_wait();
    const RansGpuEncJob& jb = jobs.j[blockIdx.x];
    const int lane = threadIdx.x;
    const int ecp = jb.ecp;
    __shared__ const uint8_t* s_ptr[kMaxEcParallel];
    __shared__ int s_size[kMaxEcParallel];
    __shared__ int s_bad;
    __shared__ int s_pos[kMaxEcParallel / 2 + 1], s_na[kMaxEcParallel / 2], s_nb[kMaxEcParallel / 2];
    __shared__ int s_total;
    if (lane == 0) {
        s_bad = 0;
    }
    __syncwarp();
    if (lane < ecp) {
        int off = 0;
        for (int i = 0; i < lane; ++i) {
            off += lane_cap(jb.n_y, jb.n_z, ecp, i);
        }
        const int cap = lane_cap(jb.n_y, jb.n_z, ecp, lane);
        Writer w{jb.scratch + off, cap, kRansL, false, false};
        int b, e;
        split(jb.n_y, ecp, lane, &b, &e);
        const uint32_t* yenc = t.enc[1];
        for (int k = e - 1; k >= b; --k) {
            const int16_t c = __ldg(jb.y + k);
            const int idx = c & 0xff;
            if (idx >= t.count[1]) {
                atomicExch(&s_bad, kRansGpuBadIndex);
                break;
            }
            w.symbol(static_cast<int8_t>(c >> 8), __ldg(t.maxv[1] + idx),
                     yenc + static_cast<size_t>(idx) * t.stride[1]);
        }
        split(jb.n_z, ecp, lane, &b, &e);
        for (int k = e - 1; k >= b; --k) {
            const int tz = (k % jb.z_ch) + jb.z_offset;
            w.symbol(__ldg(jb.z + k), __ldg(t.maxv[0] + tz),
                     t.enc[0] + static_cast<size_t>(tz) * t.stride[0]);
        }
        for (int k = 3; k >= 0; --k) {
            w.byte(w.x >> (8 * k));
        }
        if (w.overflow) {
            atomicExch(&s_bad, kRansGpuOverflow);
        }
        if (w.zero_freq) {
            atomicExch(&s_bad, kRansGpuZeroFreq);
        }
        s_ptr[lane] = w.base + w.pos;
        s_size[lane] = cap - w.pos;
    }
    __syncwarp();
    if (s_bad != 0) {
        if (lane == 0) {
            *jb.status = s_bad;
            *jb.out_size = 0;
        }
        return;
    }
    // the container (py_rans.cpp:156-249): sub-stream pairs merged as forward + reversed with
    // their shared trailing bytes overlapped, an int32 offset header in front
    const int pairs = ecp / 2;
    const bool tail = (ecp % 2) != 0;
    const int noff = ecp == 1 ? 0 : pairs - 1 + (tail ? 1 : 0);
    if (lane == 0) {
        int pos = 4 * noff;
        int32_t cum = 0;
        for (int p = 0; p < pairs; ++p) {
            const int same = shared_tail(s_ptr[2 * p], s_size[2 * p], s_ptr[2 * p + 1], s_size[2 * p + 1]);
            const int g = s_size[2 * p] + s_size[2 * p + 1] - same;
            s_pos[p] = pos;
            s_na[p] = s_size[2 * p];
            s_nb[p] = s_size[2 * p + 1] - same;
            pos += g;
            cum += g;
            if (p < noff && pos <= jb.out_cap) {
                put_i32(jb.out + 4 * p, cum);
            }
        }
        if (ecp == 1) {
            s_pos[0] = 0;
            pos = s_size[0];
        } else if (tail) {
            if (4 * (noff - 1) + 4 <= jb.out_cap) {
                put_i32(jb.out + 4 * (noff - 1), cum);
            }
            s_pos[pairs] = pos;
            pos += s_size[ecp - 1];
        }
        s_total = pos;
    }
    __syncwarp();
    if (s_total > jb.out_cap) {
        if (lane == 0) {
            *jb.status = kRansGpuOverflow;
            *jb.out_size = 0;
        }
        return;
    }
    if (ecp == 1) {
        for (int j = lane; j < s_size[0]; j += 32) {
            jb.out[j] = s_ptr[0][j];
        }
    } else {
        for (int p = 0; p < pairs; ++p) {
            uint8_t* o = jb.out + s_pos[p];
            const uint8_t* a = s_ptr[2 * p];
            const uint8_t* bb = s_ptr[2 * p + 1];
            const int na = s_na[p], nb = s_nb[p];
            for (int j = lane; j < na; j += 32) {
                o[j] = a[j];
            }
            for (int j = lane; j < nb; j += 32) {
                o[na + j] = bb[nb - 1 - j];
            }
        }
        if (tail) {
            uint8_t* o = jb.out + s_pos[pairs];
            for (int j = lane; j < s_size[ecp - 1]; j += 32) {
                o[j] = s_ptr[ecp - 1][j];
            }
        }
    }
    if (lane == 0) {
        *jb.out_size = s_total;
        *jb.status = kRansGpuOk;
    }
}

// A sub-stream reader: forward, or backwards over a pair's shared group.
struct Reader {
    const uint8_t* p;
    int left;
    int step;
    bool overrun;

    __device__ uint32_t next()
    {
        if (left <= 0) {
            overrun = true;
            return 0;
        }
        const uint32_t b = *p;
        p += step;
        --left;
        return b;
    }
};

__device__ uint32_t rd_bits(uint32_t& x, Reader& r)
{
    const uint32_t v = x & kBypassMax;
    x >>= 2;
    if (x < kRansL) {
        x = (x << 8) | r.next();
    }
    return v;
}

// rd_symbol of rans_coder.cpp (rans.cpp:108-142): linear CDF search, then the bypass digits.
__device__ int8_t rd_symbol(uint32_t& x, Reader& r, const int32_t* cdf, int32_t maxv, int last)
{
    const uint32_t cum = x & ((1u << kScaleBits) - 1);
    int s = 1;
    while (s < last && static_cast<uint32_t>(__ldg(cdf + s)) <= cum) {
        ++s;
    }
    --s;
    const uint32_t start = static_cast<uint32_t>(__ldg(cdf + s));
    const uint32_t freq = static_cast<uint32_t>(__ldg(cdf + s + 1)) - start;
    x = freq * (x >> kScaleBits) + (x & ((1u << kScaleBits) - 1)) - start;
    while (x < kRansL && !r.overrun) {
        x = (x << 8) | r.next();
    }
    int32_t v = s;
    if (v == maxv) {
        int32_t b = static_cast<int32_t>(rd_bits(x, r));
        int32_t digits = b;
        while (b == static_cast<int32_t>(kBypassMax) && digits < 64) {
            b = static_cast<int32_t>(rd_bits(x, r));
            digits += b;
        }
        int32_t raw = 0;
        for (int j = 0; j < digits; ++j) {
            const int32_t d = static_cast<int32_t>(rd_bits(x, r));
            if (j < 16) {
                raw |= d << (2 * j);
            }
        }
        v = raw + maxv;
    }
    return static_cast<int8_t>((v % 2 == 1) ? (v + 1) / 2 : -(v + 1) / 2);
}

__device__ int32_t get_i32(const uint8_t* p)
{
    uint32_t v = 0;
    for (int k = 0; k < 4; ++k) {
        v |= static_cast<uint32_t>(p[k]) << (8 * k);
    }
    return static_cast<int32_t>(v);
}

__global__ void __launch_bounds__(32) rans_gpu_decode_kernel(RansGpuTables t, DecJobs jobs)
{
    griddep_launch_dependents();
    griddep_wait();
    const RansGpuDecJob& jb = jobs.j[blockIdx.x];
    const int lane = threadIdx.x;
    const int ecp = jb.ecp;
    __shared__ int s_status;
    if (lane == 0) {
        s_status = 0;
    }
    __syncwarp();
    if (lane < ecp) {
        Reader r{jb.data, jb.size, 1, false};
        bool ok = true;
        if (ecp > 1) {
            const int pairs = ecp / 2;
            const bool tail = (ecp % 2) != 0;
            const int noff = pairs - 1 + (tail ? 1 : 0);
            int32_t off[kMaxEcParallel];
            ok = jb.size >= 4 * noff;
            const int pay_n = jb.size - 4 * noff;
            int prev = 0;
            for (int k = 0; ok && k < noff; ++k) {
                off[k] = get_i32(jb.data + 4 * k);
                ok = off[k] >= prev && off[k] <= pay_n;
                prev = off[k];
            }
            if (ok) {
                const uint8_t* pay = jb.data + 4 * noff;
                if (tail && lane == ecp - 1) {
                    r = Reader{pay + off[noff - 1], pay_n - off[noff - 1], 1, false};
                } else {
                    const int p = lane / 2;
                    const int g0 = (p == 0) ? 0 : off[p - 1];
                    const int g1 = (p < noff) ? off[p] : (tail ? off[noff - 1] : pay_n);
                    r = (lane % 2 == 0) ? Reader{pay + g0, g1 - g0, 1, false}
                                        : Reader{pay + g1 - 1, g1 - g0, -1, false};
                }
            }
        }
        if (!ok) {
            atomicExch(&s_status, kRansGpuBadHeader);
        } else {
            uint32_t x = 0;
            for (int k = 0; k < 4; ++k) {
                x |= r.next() << (8 * k);
            }
            int b, e;
            split(jb.n_z, ecp, lane, &b, &e);
            const int zlast = t.stride[0] - 1;
            for (int k = b; k < e; ++k) {
                const int tz = (k % jb.z_ch) + jb.z_offset;
                jb.z_out[k] = rd_symbol(x, r, t.cdf[0] + static_cast<size_t>(tz) * t.stride[0],
                                        __ldg(t.maxv[0] + tz), zlast);
            }
            split(jb.n_y, ecp, lane, &b, &e);
            const int ylast = t.stride[1] - 1;
            for (int k = b; k < e; ++k) {
                const int ty = __ldg(jb.y_idx + k);
                if (ty >= t.count[1]) {
                    atomicExch(&s_status, kRansGpuBadIndex);
                    break;
                }
                jb.y_out[k] = rd_symbol(x, r, t.cdf[1] + static_cast<size_t>(ty) * t.stride[1],
                                        __ldg(t.maxv[1] + ty), ylast);
            }
            if (r.overrun) {
                atomicExch(&s_status, kRansGpuOverrun);
            }
        }
    }
    __syncwarp();
    if (lane == 0) {
        *jb.status = s_status;
    }
}

}  // namespace

size_t rans_gpu_scratch_bytes(int n_y, int n_z, int ecp)
{
    if (ecp < 1 || ecp > kMaxEcParallel || n_y < 0 || n_z < 0) {
        return 0;
    }
    size_t total = 0;
    for (int i = 0; i < ecp; ++i) {
        total += static_cast<size_t>(lane_cap(n_y, n_z, ecp, i));
    }
    return total;
}

cudaError_t rans_gpu_upload(const RansTables& tables, RansGpuTables* out, void** storage)
{
    *storage = nullptr;
    if (!tables.ready()) {
        return cudaErrorInvalidValue;
    }
    const RansTable* set[2] = {&tables.z(), &tables.y()};
    size_t bytes = 0;
    for (const RansTable* s : set) {
        bytes += (s->enc.size() + s->cdf.size() + s->max_value.size()) * 4 + 3 * 256;
    }
    uint8_t* base = nullptr;
    cudaError_t e = cudaMalloc(&base, bytes);
    if (e != cudaSuccess) {
        return e;
    }
    size_t pos = 0;
    auto put = [&](const void* src, size_t n) {
        uint8_t* dst = base + pos;
        pos += (n + 255) / 256 * 256;
        if (n > 0 && cudaMemcpy(dst, src, n, cudaMemcpyHostToDevice) != cudaSuccess) {
            e = cudaErrorMemoryAllocation;
        }
        return dst;
    };
    for (int i = 0; i < 2; ++i) {
        const RansTable& s = *set[i];
        out->enc[i] = reinterpret_cast<const uint32_t*>(put(s.enc.data(), s.enc.size() * 4));
        out->cdf[i] = reinterpret_cast<const int32_t*>(put(s.cdf.data(), s.cdf.size() * 4));
        out->maxv[i] = reinterpret_cast<const int32_t*>(put(s.max_value.data(), s.max_value.size() * 4));
        out->count[i] = s.count;
        out->stride[i] = s.stride;
    }
    if (e != cudaSuccess) {
        cudaFree(base);
        return e;
    }
    *storage = base;
    return cudaSuccess;
}

cudaError_t launch_rans_gpu_encode(const RansGpuTables& t, const RansGpuEncJob* jobs, int njobs,
                                   cudaStream_t s)
{
    if (njobs < 1 || njobs > kRansGpuMaxJobs || jobs == nullptr || t.count[0] == 0 ||
        t.count[1] == 0) {
        return cudaErrorInvalidValue;
    }
    EncJobs pj;
    for (int i = 0; i < njobs; ++i) {
        const RansGpuEncJob& j = jobs[i];
        if (j.ecp < 1 || j.ecp > kMaxEcParallel || j.n_y < 0 || j.n_z < 0 ||
            (j.n_y > 0 && j.y == nullptr) || (j.n_z > 0 && (j.z == nullptr || j.z_ch < 1 ||
                                                          j.z_offset < 0 ||
                                                          j.z_offset + j.z_ch > t.count[0])) ||
            j.scratch == nullptr || j.out == nullptr || j.out_size == nullptr ||
            j.status == nullptr) {
            return cudaErrorInvalidValue;
        }
        pj.j[i] = j;
    }
    return launch_pdl(rans_gpu_encode_kernel, dim3(njobs), dim3(32), 0, s, t, pj);
}

cudaError_t launch_rans_gpu_decode(const RansGpuTables& t, const RansGpuDecJob* jobs, int njobs,
                                   cudaStream_t s)
{
    if (njobs < 1 || njobs > kRansGpuMaxJobs || jobs == nullptr || t.count[0] == 0 ||
        t.count[1] == 0) {
        return cudaErrorInvalidValue;
    }
    DecJobs pj;
    for (int i = 0; i < njobs; ++i) {
        const RansGpuDecJob& j = jobs[i];
        if (j.ecp < 1 || j.ecp > kMaxEcParallel || j.size < 0 || (j.size > 0 && j.data == nullptr) ||
            j.n_y < 0 || j.n_z < 0 || (j.n_y > 0 && (j.y_idx == nullptr || j.y_out == nullptr)) ||
            (j.n_z > 0 && (j.z_out == nullptr || j.z_ch < 1 || j.z_offset < 0 ||
                           j.z_offset + j.z_ch > t.count[0])) ||
            j.status == nullptr) {
            return cudaErrorInvalidValue;
        }
        pj.j[i] = j;
    }
    return launch_pdl(rans_gpu_decode_kernel, dim3(njobs), dim3(32), 0, s, t, pj);
}

}  // namespace dcvc
