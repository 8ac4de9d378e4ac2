// dense3D accepted-state frames encoded on the device: the JSON line of
// write_dense3d_frame (src/dense3d_sequence.rs:412-564) for a resident state,
// and a bounded frame stream with the output side of Dense3dSequence
// (src/dense3d_sequence.rs:42-120, 224-341): limits, byte budget, terminal
// errors.
//
// Number text. Rust's `{:.9e}` (the f32 fields) and `{:.17e}` (the f64
// fields, clocks and diagnostics) print the exact binary value rounded to
// P = 10 / 18 significant decimal digits, ties to even, as
// [-]d.ddd...e<exponent> (exponent in plain decimal: "e0", "e-3", "e21"; -0.0
// keeps its sign). For x = m 2^e2 the encoder estimates the decimal exponent
// E from the binary one, multiplies m by a 128-bit truncation of 10^k
// (k = P-1-E, pow10_table.inc) and reads the integer part I and the top 64
// fraction bits F of x 10^k from the 192-bit product. The truncation makes
// the product at most x 10^k (1 - 2^-126) below the exact value, i.e. less
// than 2^-62 below it, so only F within 8 units of one half can hide a tie or
// flip the rounding: those values (ties among them) are decided exactly by
// comparing 2 x 10^k with 2I + 1 in wide integers, as powers of 5 and 2.
//
// Kernels (one frame): k_d3_measure sizes every value of a 1024-value chunk
// from its binary exponent and a table of the first value of each printed
// exponent (exp_thresholds.inc), without forming digits, and reduces the
// chunk's text length; k_d3_scan turns the
// chunk lengths into offsets; k_d3_write formats the chunk again, places each
// thread's text in shared memory at its scanned offset and copies the chunk
// to the output with word stores. Validation (the preflight of
// src/dense3d_sequence.rs:431-455) happens in k_d3_measure; k_d3_write writes
// nothing when it failed, so a rejected frame leaves no bytes.
#include <errno.h>
#include <unistd.h>

#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>

#include "internal.hpp"

namespace rb200 {
namespace {

struct Pow10Entry {
    unsigned long long hi, lo;
    int s;
};
constexpr int kPow10Min = -300;
const Pow10Entry kPow10Host[] = {
#include "pow10_table.inc"
};
__device__ const Pow10Entry kPow10Dev[] = {
#include "pow10_table.inc"
};
constexpr int kPow10Count = int(sizeof(kPow10Host) / sizeof(kPow10Host[0]));

// Printed-exponent thresholds (exp_thresholds.inc): entry E - MIN is the bit
// pattern of the first positive value whose P-digit rounding reaches 10^E.
#include "exp_thresholds.inc"
const unsigned long long kThr64Host[] = {KEXPTHR64_LIST};
__device__ const unsigned long long kThr64Dev[] = {KEXPTHR64_LIST};
const unsigned long long kThr32Host[] = {KEXPTHR32_LIST};
__device__ const unsigned long long kThr32Dev[] = {KEXPTHR32_LIST};

template <int P>
__host__ __device__ __forceinline__ unsigned long long exp_threshold(int e) {
    if (P == 18) {
        const int i = e - KEXPTHR64_MIN;
#ifdef __CUDA_ARCH__
        return __ldg(&kThr64Dev[i]);
#else
        return kThr64Host[i];
#endif
    }
    const int i = e - KEXPTHR32_MIN;
#ifdef __CUDA_ARCH__
    return __ldg(&kThr32Dev[i]);
#else
    return kThr32Host[i];
#endif
}

__host__ __device__ __forceinline__ Pow10Entry pow10_entry(int k) {
    int i = k - kPow10Min;
    i = i < 0 ? 0 : (i >= kPow10Count ? kPow10Count - 1 : i);
#ifdef __CUDA_ARCH__
    return Pow10Entry{__ldg(&kPow10Dev[i].hi), __ldg(&kPow10Dev[i].lo), __ldg(&kPow10Dev[i].s)};
#else
    return kPow10Host[i];
#endif
}

__host__ __device__ __forceinline__ void mul64(uint64_t a, uint64_t b, uint64_t& lo, uint64_t& hi) {
#ifdef __CUDA_ARCH__
    lo = a * b;
    hi = __umul64hi(a, b);
#else
    const unsigned __int128 p = (unsigned __int128)a * b;
    lo = uint64_t(p);
    hi = uint64_t(p >> 64);
#endif
}

__host__ __device__ __forceinline__ int clz64(uint64_t v) {
#ifdef __CUDA_ARCH__
    return __clzll((long long)v);
#else
    return __builtin_clzll(v);
#endif
}

__host__ __device__ constexpr uint64_t pow10c(int n) { return n == 0 ? 1ull : 10ull * pow10c(n - 1); }

// Unsigned integer of up to 960 bits (little-endian 32-bit limbs), for the
// exact decision of near-ties only.
struct Wide {
    static constexpr int W = 30;
    uint32_t w[W];
    int n;
    __host__ __device__ void set(uint64_t lo, uint32_t hi = 0u) {
        for (int i = 0; i < W; ++i) w[i] = 0u;
        w[0] = uint32_t(lo);
        w[1] = uint32_t(lo >> 32);
        w[2] = hi;
        n = 3;
    }
    __host__ __device__ void mul(uint32_t f) {
        uint64_t carry = 0;
        for (int i = 0; i < n; ++i) {
            const uint64_t t = uint64_t(w[i]) * f + carry;
            w[i] = uint32_t(t);
            carry = t >> 32;
        }
        if (carry && n < W) w[n++] = uint32_t(carry);
    }
    __host__ __device__ void mul_pow5(int k) {
        for (; k >= 13; k -= 13) mul(1220703125u);  // 5^13
        uint32_t f = 1u;
        for (; k > 0; --k) f *= 5u;
        mul(f);
    }
    __host__ __device__ void shl(int b) {
        const int q = b >> 5, r = b & 31;
        int m = n + q + 1;
        if (m > W) m = W;
        for (int i = m - 1; i >= 0; --i) {
            const int s = i - q;
            const uint32_t hi = (s >= 0 && s < n) ? w[s] : 0u;
            const uint32_t lo = (s >= 1 && s - 1 < n) ? w[s - 1] : 0u;
            w[i] = r ? (hi << r) | (lo >> (32 - r)) : hi;
        }
        n = m;
    }
};

__host__ __device__ int wide_cmp(const Wide& a, const Wide& b) {
    const int n = a.n > b.n ? a.n : b.n;
    for (int i = n - 1; i >= 0; --i) {
        const uint32_t x = i < a.n ? a.w[i] : 0u, y = i < b.n ? b.w[i] : 0u;
        if (x != y) return x < y ? -1 : 1;
    }
    return 0;
}

// Sign of 2 m 2^e2 10^k - (2I + 1): with 10^k = 5^k 2^k both sides are
// integers after moving the powers of 5 and of 2 to one side each. The
// operands stay below 2^900 for every finite double (at most 53 bits of m
// times 5^343, or 65 bits of 2I + 1 times 5^300).
__host__ __device__ __noinline__ int exact_cmp(uint64_t m, int e2, int k, uint64_t I) {
    Wide a, b;
    a.set(m);
    b.set(2 * I + 1, uint32_t(I >> 63));
    if (k >= 0)
        a.mul_pow5(k);
    else
        b.mul_pow5(-k);
    const int t = e2 + k + 1;
    if (t >= 0)
        a.shl(t);
    else
        b.shl(-t);
    return wide_cmp(a, b);
}

struct Dec {
    uint64_t n;  // P significant digits (0 for a zero)
    int e;       // decimal exponent of the first digit
};

// x = m 2^e2 (m > 0) rounded to P significant digits, ties to even.
template <int P>
__host__ __device__ Dec to_decimal(uint64_t m, int e2) {
    constexpr uint64_t LO = pow10c(P - 1), HI = pow10c(P);
    const int L = e2 + 63 - clz64(m);  // floor(log2 x)
    int E = (L * 78913) >> 18;         // floor(L log10 2): E or E - 1
    for (int attempt = 0; attempt < 4; ++attempt) {
        const int k = (P - 1) - E;
        const Pow10Entry t = pow10_entry(k);
        uint64_t l0, h0, l1, h1;
        mul64(m, t.lo, l0, h0);
        mul64(m, t.hi, l1, h1);
        const uint64_t w0 = l0, w1 = h0 + l1, w2 = h1 + (w1 < l1 ? 1u : 0u);
        const int s1 = -(e2 + t.s) - 64;  // integer part = product >> (64 + s1)
        if (s1 < 0) {
            E += 1;
            continue;
        }
        if (s1 > 63) {
            E -= 1;
            continue;
        }
        if (s1 ? (w2 >> s1) != 0 : w2 != 0) {
            E += 1;
            continue;
        }
        const uint64_t I = s1 ? (w1 >> s1) | (w2 << (64 - s1)) : w1;
        const uint64_t F = s1 ? (w0 >> s1) | (w1 << (64 - s1)) : w0;
        if (I >= HI) {
            E += 1;
            continue;
        }
        constexpr uint64_t half = 1ull << 63;
        uint64_t N;
        if (F > half)
            N = I + 1;
        else if (F < half - 8)
            N = I;
        else {
            const int c = exact_cmp(m, e2, k, I);
            N = c < 0 ? I : (c > 0 ? I + 1 : I + (I & 1u));
        }
        if (N < LO) {  // fewer than P digits even after rounding: E was one too high
            E -= 1;
            continue;
        }
        if (N == HI) {
            N = LO;
            E += 1;
        }
        return Dec{N, E};
    }
    return Dec{0, 0};
}

__host__ __device__ __forceinline__ uint64_t bits_of(double x) {
#ifdef __CUDA_ARCH__
    return uint64_t(__double_as_longlong(x));
#else
    uint64_t b;
    std::memcpy(&b, &x, 8);
    return b;
#endif
}
__host__ __device__ __forceinline__ uint32_t bits_of(float x) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(x);
#else
    uint32_t b;
    std::memcpy(&b, &x, 4);
    return b;
#endif
}

// A value ready for its text: sign and rounded digits.
struct Num {
    Dec d;
    bool neg;
};

__host__ __device__ __forceinline__ Num num64(double x) {
    const uint64_t b = bits_of(x);
    const int be = int((b >> 52) & 0x7ff);
    uint64_t m = b & ((1ull << 52) - 1);
    int e2 = -1074;
    if (be) {
        m |= 1ull << 52;
        e2 = be - 1075;
    }
    return Num{m ? to_decimal<18>(m, e2) : Dec{0, 0}, (b >> 63) != 0};
}
__host__ __device__ __forceinline__ Num num32(float x) {
    const uint32_t b = bits_of(x);
    const int be = int((b >> 23) & 0xff);
    uint64_t m = b & 0x7fffffu;
    int e2 = -149;
    if (be) {
        m |= 1u << 23;
        e2 = be - 150;
    }
    return Num{m ? to_decimal<10>(m, e2) : Dec{0, 0}, (b >> 31) != 0};
}

// Length of the text of a value with magnitude bits `abs` (a positive
// finite value, or zero) without forming its digits: the printed exponent is
// the binary estimate E (E <= floor(log10 x)) raised by the thresholds it
// reaches (at most two).
template <int P>
__host__ __device__ __forceinline__ int text_len_bits(unsigned long long abs, int mant_bits, int bias, int sub_e2,
                                                      bool neg) {
    int e = 0;
    if (abs) {
        const int be = int(abs >> mant_bits);
        const int L = be ? be - bias : sub_e2 + 63 - clz64(abs);  // floor(log2 x)
        const int E = (L * 78913) >> 18;
        e = E + int(abs >= exp_threshold<P>(E + 1)) + int(abs >= exp_threshold<P>(E + 2));
    }
    const int ae = e < 0 ? -e : e;
    return int(neg) + P + 2 + int(e < 0) + (ae >= 100 ? 3 : (ae >= 10 ? 2 : 1));
}
__host__ __device__ __forceinline__ int len64(double x) {
    const uint64_t b = bits_of(x);
    return text_len_bits<18>(b & 0x7fffffffffffffffull, 52, 1023, -1074, (b >> 63) != 0);
}
__host__ __device__ __forceinline__ int len32(float x) {
    const uint32_t b = bits_of(x);
    return text_len_bits<10>(b & 0x7fffffffu, 23, 127, -149, (b >> 31) != 0);
}

template <int P>
__host__ __device__ __forceinline__ int text_len(const Num& v) {
    const int ae = v.d.e < 0 ? -v.d.e : v.d.e;
    return int(v.neg) + P + 2 + int(v.d.e < 0) + (ae >= 100 ? 3 : (ae >= 10 ? 2 : 1));
}

// [-]d.ddd...e[-]x; returns the length.
template <int P>
__host__ __device__ __forceinline__ int text_put(const Num& v, char* out) {
    char dig[P];
    uint32_t lo = uint32_t(v.d.n % 1000000000ull);
    uint32_t hi = uint32_t(v.d.n / 1000000000ull);
#pragma unroll
    for (int i = P - 1; i >= P - 9; --i) {
        dig[i] = char('0' + lo % 10u);
        lo /= 10u;
    }
#pragma unroll
    for (int i = P - 10; i >= 0; --i) {
        dig[i] = char('0' + hi % 10u);
        hi /= 10u;
    }
    int p = 0;
    if (v.neg) out[p++] = '-';
    out[p++] = dig[0];
    out[p++] = '.';
#pragma unroll
    for (int i = 1; i < P; ++i) out[p++] = dig[i];
    out[p++] = 'e';
    int e = v.d.e;
    if (e < 0) {
        out[p++] = '-';
        e = -e;
    }
    if (e >= 100) out[p++] = char('0' + e / 100);
    if (e >= 10) out[p++] = char('0' + (e / 10) % 10);
    out[p++] = char('0' + e % 10);
    return p;
}

// ------------------------------------------------------------ device encoder
constexpr int D3_THREADS = 256;
constexpr int D3_VPT = 4;
constexpr int D3_CHUNK = D3_THREADS * D3_VPT;
constexpr int D3_MAX_TEXT = 26;       // longest value text plus its comma
constexpr int D3_MAX_JOINERS = 2048;  // all joiner strings of a frame together
constexpr int D3_STAGE = D3_CHUNK * D3_MAX_TEXT + D3_MAX_JOINERS;

enum : unsigned { BAD_VELOCITY = 1u, BAD_CELL = 2u };

struct D3Status {
    unsigned bad;
    unsigned pad;
    unsigned long long text;  // bytes of all values and joiners (the line minus its header)
};

struct D3Args {
    const void* field[6];             // velocity x, y, z, tracer, fraction, pressure
    int vel_f64;                      // velocity arrays hold f64 (printed as the f32 they round to)
    unsigned long long end[6];        // segment s covers values [end[s-1], end[s])
    const char* strings;              // header, then joiners J0..J5 (J5 closes the line)
    int off[8];                       // header [off[0], off[1]); J_s [off[s+1], off[s+2])
    unsigned long long* block_len;
    unsigned long long* block_off;
    D3Status* status;
    char* out;
    unsigned long long capacity;
    int nblocks;
};

__device__ __forceinline__ unsigned long long block_sum_u64(unsigned long long v, unsigned long long* sm) {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) sm[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < D3_THREADS / 32 ? sm[lane] : 0ull;
#pragma unroll
        for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    }
    return v;  // valid in thread 0
}

// Text length of value i with its separator, from the exponent thresholds
// (no digits), and its preflight.
__device__ __forceinline__ int d3_len(const D3Args& a, unsigned long long i, unsigned& bad) {
    int s = 0;
#pragma unroll
    for (int q = 0; q < 5; ++q) s += i >= a.end[q] ? 1 : 0;
    const unsigned long long j = i - (s ? a.end[s - 1] : 0ull);
    int len;
    if (s < 4) {
        float x = 0.0f;
        if (s < 3)
            x = a.vel_f64 ? float(static_cast<const double*>(a.field[s])[j]) : static_cast<const float*>(a.field[s])[j];
        else if (a.field[3])
            x = static_cast<const float*>(a.field[3])[j];
        if (!isfinite(x)) bad |= s < 3 ? BAD_VELOCITY : BAD_CELL;
        len = len32(x);
    } else {
        double x = 0.0;
        if (a.field[s]) x = static_cast<const double*>(a.field[s])[j];
        if (!isfinite(x) || (s == 4 && !(x >= 0.0 && x <= 1.0))) bad |= BAD_CELL;
        len = len64(x);
    }
    return len + ((i + 1 == a.end[s]) ? a.off[s + 2] - a.off[s + 1] : 1);
}

__global__ void __launch_bounds__(D3_THREADS) k_d3_measure(D3Args a) {
    __shared__ unsigned long long sm[32];
    const unsigned long long base = (unsigned long long)blockIdx.x * D3_CHUNK + threadIdx.x * D3_VPT;
    unsigned long long len = 0;
    unsigned bad = 0u;
#pragma unroll
    for (int u = 0; u < D3_VPT; ++u) {
        const unsigned long long i = base + u;
        if (i >= a.end[5]) break;
        len += d3_len(a, i, bad);
    }
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (bad && (threadIdx.x & 31) == 0) atomicOr(&a.status->bad, bad);
    len = block_sum_u64(len, sm);
    if (threadIdx.x == 0) a.block_len[blockIdx.x] = len;
}

// Exclusive scan of the chunk lengths (one block).
__global__ void __launch_bounds__(1024) k_d3_scan(D3Args a) {
    __shared__ unsigned long long sm[32];
    const int per = (a.nblocks + 1023) / 1024;
    const int b0 = threadIdx.x * per;
    unsigned long long mine = 0;
    for (int b = b0; b < b0 + per && b < a.nblocks; ++b) mine += a.block_len[b];
    // inclusive scan of the per-thread sums
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long x = mine;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) sm[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned long long t = sm[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, t, d);
            if (lane >= d) t += y;
        }
        sm[lane] = t;
    }
    __syncthreads();
    unsigned long long run = x - mine + (warp ? sm[warp - 1] : 0ull);
    for (int b = b0; b < b0 + per && b < a.nblocks; ++b) {
        a.block_off[b] = run;
        run += a.block_len[b];
    }
    if (threadIdx.x == 1023) a.status->text = run;
}

__global__ void __launch_bounds__(D3_THREADS) k_d3_write(D3Args a) {
    __shared__ __align__(16) char stage[D3_STAGE + 16];
    __shared__ unsigned long long sm[32];
    const D3Status st = *a.status;
    const unsigned long long header = (unsigned long long)(a.off[1] - a.off[0]);
    if (st.bad || header + st.text > a.capacity) return;
    if (blockIdx.x == 0)
        for (int c = threadIdx.x; c < int(header); c += D3_THREADS) a.out[c] = a.strings[a.off[0] + c];
    const unsigned long long base = (unsigned long long)blockIdx.x * D3_CHUNK + threadIdx.x * D3_VPT;
    // lengths first (no digits), then the block's exclusive scan of them
    int mine = 0;
    unsigned bad = 0u;
#pragma unroll 1
    for (int u = 0; u < D3_VPT; ++u)
        if (base + u < a.end[5]) mine += d3_len(a, base + u, bad);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = mine;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) sm[warp] = (unsigned long long)x;
    __syncthreads();
    // the chunk's text sits in shared memory at the output's alignment
    // modulo 16, so that 16-byte words of both line up
    char* dst = a.out + header + a.block_off[blockIdx.x];
    const unsigned shift = unsigned((uintptr_t)dst & 15u);
    int before = 0;
    for (int q = 0; q < warp; ++q) before += int(sm[q]);
    int p = int(shift) + before + x - mine;
    // the digits, one value at a time (one copy of the code for both types)
#pragma unroll 1
    for (int u = 0; u < D3_VPT; ++u) {
        const unsigned long long i = base + u;
        if (i >= a.end[5]) break;
        int s = 0;
#pragma unroll
        for (int q = 0; q < 5; ++q) s += i >= a.end[q] ? 1 : 0;
        const unsigned long long j = i - (s ? a.end[s - 1] : 0ull);
        if (s < 4) {
            float v = 0.0f;
            if (s < 3)
                v = a.vel_f64 ? float(static_cast<const double*>(a.field[s])[j])
                              : static_cast<const float*>(a.field[s])[j];
            else if (a.field[3])
                v = static_cast<const float*>(a.field[3])[j];
            p += text_put<10>(num32(v), stage + p);
        } else {
            const double v = a.field[s] ? static_cast<const double*>(a.field[s])[j] : 0.0;
            p += text_put<18>(num64(v), stage + p);
        }
        if (i + 1 == a.end[s]) {
            for (int c = a.off[s + 1]; c < a.off[s + 2]; ++c) stage[p++] = a.strings[c];
        } else {
            stage[p++] = ',';
        }
    }
    __syncthreads();
    // the chunk's text: bytes up to a 16-byte boundary of the output, 16-byte
    // words, the tail bytes
    const unsigned L = unsigned(a.block_len[blockIdx.x]);
    const char* src = stage + shift;
    const unsigned head = min(L, (16u - shift) & 15u);
    if (threadIdx.x < head) dst[threadIdx.x] = src[threadIdx.x];
    const unsigned words = (L - head) >> 4;
    for (unsigned q = threadIdx.x; q < words; q += D3_THREADS)
        *reinterpret_cast<uint4*>(dst + head + 16u * q) = *reinterpret_cast<const uint4*>(src + head + 16u * q);
    const unsigned tail = head + 16u * words;
    if (threadIdx.x < L - tail) dst[tail + threadIdx.x] = src[tail + threadIdx.x];
}

// ------------------------------------------------------------ host text
void put_f64(std::string& s, double v) {
    char buf[32];
    const int n = text_put<18>(num64(v), buf);
    s.append(buf, size_t(n));
}

const char* const kFieldNames[6] = {"velocity_x", "velocity_y", "velocity_z", "tracer", "fraction", "pressure"};

// Preflight of the clocks and report (src/dense3d_sequence.rs:456-494).
bool frame_info_ok(const rb200_dense3d_frame& f) {
    if (!std::isfinite(f.time_s)) return false;
    if (f.has_diagnostics) {
        if (!(std::isfinite(f.dt_s) && f.dt_s > 0.0)) return false;
        const double d[11] = {f.pressure_residual_m3_s2, f.carrier_divergence_s_inv, f.liquid_divergence_s_inv,
                              f.volume_before_m3,        f.volume_after_m3,          f.mass_after_kg,
                              f.inward_m3,               f.outward_m3,               f.source_m3,
                              f.balance_m3,              f.rounding_budget_m3};
        for (double x : d)
            if (!std::isfinite(x)) return false;
        return true;
    }
    return f.frame == 0 && f.time_s == 0.0 && f.carrier_stamp_version == 0;
}

// The frame's constant text: header (up to the first '[') and the joiners.
std::string frame_strings(const rb200_dense3d_frame& f, int off[8]) {
    std::string s;
    off[0] = 0;
    s += "{\"frame\":" + std::to_string(f.frame) + ",\"time_s\":";
    put_f64(s, f.time_s);
    s += ",\"dt_s\":";
    put_f64(s, f.has_diagnostics ? f.dt_s : 0.0);
    s += ",\"carrier_stamp\":{\"id\":\"" + std::to_string(f.carrier_stamp_id) + "\",\"version\":\"" +
         std::to_string(f.carrier_stamp_version) + "\"},\"liquid_stamp\":{\"id\":\"" +
         std::to_string(f.liquid_stamp_id) + "\",\"version\":\"" + std::to_string(f.liquid_stamp_version) +
         "\"},\"fields\":{\"velocity_x\":[";
    off[1] = int(s.size());
    for (int q = 0; q < 5; ++q) {
        s += std::string("],\"") + kFieldNames[q + 1] + "\":[";
        off[q + 2] = int(s.size());
    }
    s += "]},\"diagnostics\":";
    if (f.has_diagnostics) {
        static const char* names[11] = {"pressure_residual_m3_s2", "carrier_divergence_s_inv",
                                        "liquid_divergence_s_inv", "volume_before_m3",
                                        "volume_after_m3",         "mass_after_kg",
                                        "inward_m3",               "outward_m3",
                                        "source_m3",               "balance_m3",
                                        "rounding_budget_m3"};
        const double d[11] = {f.pressure_residual_m3_s2, f.carrier_divergence_s_inv, f.liquid_divergence_s_inv,
                              f.volume_before_m3,        f.volume_after_m3,          f.mass_after_kg,
                              f.inward_m3,               f.outward_m3,               f.source_m3,
                              f.balance_m3,              f.rounding_budget_m3};
        s += "{\"pressure_iterations\":" + std::to_string(f.pressure_iterations);
        for (int q = 0; q < 11; ++q) {
            s += std::string(",\"") + names[q] + "\":";
            put_f64(s, d[q]);
        }
        s += "}";
    } else {
        s += "null";
    }
    s += "}\n";
    off[7] = int(s.size());
    return s;
}

}  // namespace
}  // namespace rb200

using namespace rb200;

struct rb200_dense3d_encoder {
    int device = 0;
    unsigned long long faces[3] = {0, 0, 0};
    unsigned long long cells = 0;
    int nblocks = 0;
    char* d_strings = nullptr;
    unsigned long long* d_block = nullptr;  // [2][nblocks]
    D3Status* d_status = nullptr;
    D3Status* h_status = nullptr;  // pinned
    std::string err;
};

// The frame stream: frames are encoded on the caller's stream (the caller
// waits for the encode, a fraction of a millisecond), then copied to pinned
// host memory on the writer's own copy stream and written by the writer's
// thread, so that the copy and the write overlap the caller's next step. Two
// slots (device text, pinned text) alternate; a frame waits for its slot.
struct rb200_dense3d_writer {
    static constexpr int SLOTS = 2;
    rb200_dense3d_encoder* enc = nullptr;
    rb200_dense3d_limits limits{};
    int fd = -1;
    int device = 0;
    char* d_text[SLOTS] = {};
    char* h_text[SLOTS] = {};  // pinned
    uint64_t capacity = 0;
    cudaStream_t copy = nullptr;
    cudaEvent_t copied[SLOTS] = {};
    std::thread thread;
    std::mutex mu;
    std::condition_variable cv;
    bool busy[SLOTS] = {};
    uint64_t job_len[SLOTS] = {};
    int queue[SLOTS] = {};
    int q_head = 0, q_size = 0;
    bool stop = false;
    uint64_t frames = 0;    // frames accepted (encoded and queued)
    uint64_t reserved = 0;  // bytes of the accepted frames
    uint64_t bytes = 0;     // bytes written
    bool aborted = false;
    int async_status = 0;   // a failed copy or write, reported by the next call
    std::string err;
};

namespace {

uint64_t frame_bound(const rb200_dense3d_encoder* e) {
    const uint64_t f32s = e->faces[0] + e->faces[1] + e->faces[2] + e->cells;
    return f32s * 17u + 2u * e->cells * 26u + D3_MAX_JOINERS + 512u;
}

int encode(rb200_dense3d_encoder* e, const rb200_dense3d_frame* f, const rb200_dense3d_fields* fl, char* out,
           uint64_t capacity, uint64_t* length, cudaStream_t s) {
    if (!frame_info_ok(*f)) {
        e->err = "dense3D export: InvalidState(\"state clock/stamp or report\")";
        return RB200_DENSE3D_INVALID_STATE;
    }
    D3Args a{};
    a.field[0] = fl->u;
    a.field[1] = fl->v;
    a.field[2] = fl->w;
    a.field[3] = fl->tracer;
    a.field[4] = fl->fraction;
    a.field[5] = fl->pressure;
    a.vel_f64 = fl->velocity_storage == RB200_FACES_F64;
    unsigned long long run = 0;
    for (int q = 0; q < 6; ++q) {
        run += q < 3 ? e->faces[q] : e->cells;
        a.end[q] = run;
    }
    const std::string str = frame_strings(*f, a.off);
    if (a.off[7] - a.off[1] > D3_MAX_JOINERS) {
        e->err = "dense3D frame: joiner text too long";
        return RB200_INVALID_ARGUMENT;
    }
    RB200_CUDA(cudaMemcpyAsync(e->d_strings, str.data(), str.size(), cudaMemcpyHostToDevice, s));
    RB200_CUDA(cudaMemsetAsync(e->d_status, 0, sizeof(D3Status), s));
    a.strings = e->d_strings;
    a.block_len = e->d_block;
    a.block_off = e->d_block + e->nblocks;
    a.status = e->d_status;
    a.out = out;
    a.capacity = capacity;
    a.nblocks = e->nblocks;
    k_d3_measure<<<e->nblocks, D3_THREADS, 0, s>>>(a);
    k_d3_scan<<<1, 1024, 0, s>>>(a);
    k_d3_write<<<e->nblocks, D3_THREADS, 0, s>>>(a);
    RB200_CUDA(cudaGetLastError());
    RB200_CUDA(cudaMemcpyAsync(e->h_status, e->d_status, sizeof(D3Status), cudaMemcpyDeviceToHost, s));
    RB200_CUDA(cudaStreamSynchronize(s));
    const D3Status st = *e->h_status;
    if (st.bad & BAD_VELOCITY) {
        e->err = "dense3D export: InvalidState(\"nonfinite velocity\")";
        return RB200_DENSE3D_INVALID_STATE;
    }
    if (st.bad) {
        e->err = "dense3D export: InvalidState(\"nonfinite or invalid cell field\")";
        return RB200_DENSE3D_INVALID_STATE;
    }
    *length = uint64_t(a.off[1]) + st.text;
    if (*length > capacity) {
        e->err = "dense3D frame: output buffer too small";
        return RB200_DENSE3D_LIMIT;
    }
    return RB200_OK;
}

}  // namespace

extern "C" {

int rb200_dense3d_encoder_create(const rb200_grid* grid, int device, rb200_dense3d_encoder** out) {
    if (!grid || !out) return RB200_INVALID_ARGUMENT;
    *out = nullptr;
    GridDev g;
    int rc = make_grid_dev(grid, 1.0, &g);
    if (rc) return rc;
    RB200_CUDA(cudaSetDevice(device));
    auto* e = new rb200_dense3d_encoder();
    e->device = device;
    for (int a = 0; a < 3; ++a) e->faces[a] = (unsigned long long)g.flen[a];
    e->cells = (unsigned long long)g.cells;
    const unsigned long long total = e->faces[0] + e->faces[1] + e->faces[2] + 3ull * e->cells;
    e->nblocks = int((total + D3_CHUNK - 1) / D3_CHUNK);
    if (cudaMalloc(&e->d_strings, 4096) != cudaSuccess ||
        cudaMalloc(&e->d_block, 2 * size_t(e->nblocks) * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&e->d_status, sizeof(D3Status)) != cudaSuccess ||
        cudaMallocHost(&e->h_status, sizeof(D3Status)) != cudaSuccess) {
        rb200_dense3d_encoder_destroy(e);
        cudaGetLastError();
        return RB200_OUT_OF_MEMORY;
    }
    *out = e;
    return RB200_OK;
}

void rb200_dense3d_encoder_destroy(rb200_dense3d_encoder* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    cudaFree(e->d_strings);
    cudaFree(e->d_block);
    cudaFree(e->d_status);
    cudaFreeHost(e->h_status);
    delete e;
}

uint64_t rb200_dense3d_frame_bound(const rb200_dense3d_encoder* e) { return e ? frame_bound(e) : 0; }

const char* rb200_dense3d_encoder_error(const rb200_dense3d_encoder* e) { return e ? e->err.c_str() : ""; }

int rb200_dense3d_encode(rb200_dense3d_encoder* e, const rb200_dense3d_frame* frame,
                         const rb200_dense3d_fields* fields, void* out, uint64_t capacity, uint64_t* length,
                         void* stream) {
    if (!e || !frame || !fields || !out || !length || !fields->u || !fields->v || !fields->w)
        return RB200_INVALID_ARGUMENT;
    cudaSetDevice(e->device);
    return encode(e, frame, fields, static_cast<char*>(out), capacity, length, static_cast<cudaStream_t>(stream));
}

int rb200_dense3d_text_f64(double value, char* out, size_t capacity) {
    if (!out || capacity < 26) return RB200_INVALID_ARGUMENT;
    const int n = text_put<18>(num64(value), out);
    out[n] = '\0';
    return n;
}

int rb200_dense3d_text_f32(float value, char* out, size_t capacity) {
    if (!out || capacity < 17) return RB200_INVALID_ARGUMENT;
    const int n = text_put<10>(num32(value), out);
    out[n] = '\0';
    return n;
}

// ------------------------------------------------------------ frame stream
}  // extern "C"

namespace {

// The writer's thread: waits for each queued slot's copy, writes it out.
void writer_loop(rb200_dense3d_writer* w) {
    cudaSetDevice(w->device);
    for (;;) {
        int slot;
        {
            std::unique_lock<std::mutex> lock(w->mu);
            w->cv.wait(lock, [&] { return w->q_size > 0 || w->stop; });
            if (w->q_size == 0) return;
            slot = w->queue[w->q_head];
        }
        int status = 0;
        std::string msg;
        if (cudaEventSynchronize(w->copied[slot]) != cudaSuccess) {
            status = RB200_EXECUTION;
            msg = "dense3D frame: device copy failed";
        }
        const uint64_t len = w->job_len[slot];
        uint64_t done = 0;
        while (!status && done < len) {
            const ssize_t n = ::write(w->fd, w->h_text[slot] + done, size_t(len - done));
            if (n < 0) {
                if (errno == EINTR) continue;
                status = RB200_DENSE3D_IO;
                msg = std::string("dense3D export: Io(") + std::strerror(errno) + ")";
                break;
            }
            done += uint64_t(n);
            std::lock_guard<std::mutex> lock(w->mu);
            w->bytes += uint64_t(n);
        }
        std::lock_guard<std::mutex> lock(w->mu);
        if (status && !w->async_status) {
            w->async_status = status;
            w->err = msg;
        }
        w->busy[slot] = false;
        w->q_head = (w->q_head + 1) % rb200_dense3d_writer::SLOTS;
        w->q_size -= 1;
        w->cv.notify_all();
    }
}

// Wait until every queued frame is written; a failure seen by the thread is
// terminal. Called without the lock.
int drain(rb200_dense3d_writer* w) {
    std::unique_lock<std::mutex> lock(w->mu);
    w->cv.wait(lock, [&] { return w->q_size == 0; });
    if (w->async_status) {
        w->aborted = true;
        return w->async_status;
    }
    return RB200_OK;
}

}  // namespace

extern "C" {

int rb200_dense3d_writer_create(const rb200_grid* grid, const rb200_dense3d_limits* limits, int fd, int device,
                                rb200_dense3d_writer** out) {
    if (!grid || !limits || !out || fd < 0) return RB200_INVALID_ARGUMENT;
    *out = nullptr;
    // Dense3dSequence::new (src/dense3d_sequence.rs:90-100)
    uint64_t cells = grid->counts[0] * grid->counts[1] * grid->counts[2];
    if (limits->max_frames == 0 || limits->max_bytes == 0 || cells > limits->max_cells) {
        set_error("dense3D export: Limit");
        return RB200_DENSE3D_LIMIT;
    }
    rb200_dense3d_encoder* e = nullptr;
    int rc = rb200_dense3d_encoder_create(grid, device, &e);
    if (rc) return rc;
    auto* w = new rb200_dense3d_writer();
    w->enc = e;
    w->limits = *limits;
    w->fd = fd;
    w->device = device;
    w->capacity = frame_bound(e);
    bool ok = cudaStreamCreateWithFlags(&w->copy, cudaStreamNonBlocking) == cudaSuccess;
    for (int k = 0; ok && k < rb200_dense3d_writer::SLOTS; ++k)
        ok = cudaMalloc(&w->d_text[k], w->capacity) == cudaSuccess &&
             cudaMallocHost(&w->h_text[k], w->capacity) == cudaSuccess &&
             cudaEventCreateWithFlags(&w->copied[k], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        rb200_dense3d_writer_destroy(w);
        cudaGetLastError();
        return RB200_OUT_OF_MEMORY;
    }
    w->thread = std::thread(writer_loop, w);
    *out = w;
    return RB200_OK;
}

void rb200_dense3d_writer_destroy(rb200_dense3d_writer* w) {
    if (!w) return;
    if (w->thread.joinable()) {
        drain(w);
        {
            std::lock_guard<std::mutex> lock(w->mu);
            w->stop = true;
        }
        w->cv.notify_all();
        w->thread.join();
    }
    cudaSetDevice(w->device);
    for (int k = 0; k < rb200_dense3d_writer::SLOTS; ++k) {
        cudaFree(w->d_text[k]);
        cudaFreeHost(w->h_text[k]);
        if (w->copied[k]) cudaEventDestroy(w->copied[k]);
    }
    if (w->copy) cudaStreamDestroy(w->copy);
    rb200_dense3d_encoder_destroy(w->enc);
    delete w;
}

// One accepted frame: preflight and encode on the caller's stream (waited
// for), then the copy and the write are queued. Every failure is terminal for
// the stream (src/dense3d_sequence.rs:224-341); a failed copy or write of an
// earlier frame is reported here, by flush or by sync.
int rb200_dense3d_writer_frame(rb200_dense3d_writer* w, const rb200_dense3d_frame* frame,
                               const rb200_dense3d_fields* fields, void* stream) {
    if (!w || !frame || !fields) return RB200_INVALID_ARGUMENT;
    auto fail = [&](int rc, const std::string& msg) {
        std::lock_guard<std::mutex> lock(w->mu);
        w->aborted = true;
        w->err = msg;
        return rc;
    };
    int slot;
    {
        std::unique_lock<std::mutex> lock(w->mu);
        if (w->async_status) {
            w->aborted = true;
            return w->async_status;
        }
        if (w->aborted) {
            w->err = "dense3D export: Aborted";
            return RB200_DENSE3D_ABORTED;
        }
        slot = int(w->frames % rb200_dense3d_writer::SLOTS);
        w->cv.wait(lock, [&] { return !w->busy[slot] || w->async_status; });
        if (w->async_status) {
            w->aborted = true;
            return w->async_status;
        }
    }
    if (w->frames >= w->limits.max_frames) return fail(RB200_DENSE3D_LIMIT, "dense3D export: Limit");
    if (frame->frame != w->frames)
        return fail(RB200_DENSE3D_INVALID_STATE, "dense3D export: InvalidState(\"frame order\")");
    if (!fields->u || !fields->v || !fields->w) return fail(RB200_INVALID_ARGUMENT, "dense3D frame: missing field");
    cudaSetDevice(w->device);
    uint64_t len = 0;
    const int rc = encode(w->enc, frame, fields, w->d_text[slot], w->capacity, &len, static_cast<cudaStream_t>(stream));
    if (rc) return fail(rc, w->enc->err);
    if (len > w->limits.max_bytes - w->reserved)
        return fail(RB200_DENSE3D_IO, "dense3D export: Io(dense3D byte budget exhausted)");
    if (cudaMemcpyAsync(w->h_text[slot], w->d_text[slot], len, cudaMemcpyDeviceToHost, w->copy) != cudaSuccess ||
        cudaEventRecord(w->copied[slot], w->copy) != cudaSuccess)
        return fail(RB200_EXECUTION, "dense3D frame: device copy failed");
    {
        std::lock_guard<std::mutex> lock(w->mu);
        w->busy[slot] = true;
        w->job_len[slot] = len;
        w->queue[(w->q_head + w->q_size) % rb200_dense3d_writer::SLOTS] = slot;
        w->q_size += 1;
        w->frames += 1;
        w->reserved += len;
    }
    w->cv.notify_all();
    return RB200_OK;
}

// Dense3dSequence::flush (src/dense3d_sequence.rs:332-341): every accepted
// frame written; terminal on failure.
int rb200_dense3d_writer_flush(rb200_dense3d_writer* w) {
    if (!w) return RB200_INVALID_ARGUMENT;
    {
        std::lock_guard<std::mutex> lock(w->mu);
        if (w->aborted && !w->async_status) return RB200_DENSE3D_ABORTED;
    }
    return drain(w);
}

int rb200_dense3d_writer_sync(rb200_dense3d_writer* w) {
    const int rc = rb200_dense3d_writer_flush(w);
    if (rc) return rc;
    if (::fsync(w->fd) != 0 && errno != EINVAL && errno != EROFS) {
        std::lock_guard<std::mutex> lock(w->mu);
        w->aborted = true;
        w->err = std::string("dense3D export: Io(") + std::strerror(errno) + ")";
        return RB200_DENSE3D_IO;
    }
    return RB200_OK;
}

uint64_t rb200_dense3d_writer_frames(const rb200_dense3d_writer* w) { return w ? w->frames : 0; }
uint64_t rb200_dense3d_writer_bytes(const rb200_dense3d_writer* w) {
    if (!w) return 0;
    std::lock_guard<std::mutex> lock(const_cast<rb200_dense3d_writer*>(w)->mu);
    return w->bytes;
}
int rb200_dense3d_writer_aborted(const rb200_dense3d_writer* w) {
    if (!w) return 1;
    std::lock_guard<std::mutex> lock(const_cast<rb200_dense3d_writer*>(w)->mu);
    return int(w->aborted || w->async_status);
}
const char* rb200_dense3d_writer_error(const rb200_dense3d_writer* w) { return w ? w->err.c_str() : ""; }

}  // extern "C"
