/*
 * gexs_ingest.cu — ExoMol line-list ingest on the GPU: the reader layer that
 * feeds the cross-section path (Readers/Exomol/ExomolStateReader.cpp and
 * Readers/Exomol/exomol_functions.cpp in the reference, which parse text on
 * one host thread with strtol/strtod/istream).
 *
 * A file's bytes are copied to the device once; a newline index is built
 * with two passes over 4 KiB chunks (one warp per chunk) and an exclusive
 * scan; then one thread parses one record:
 *  - .states (exomol_functions.cpp:8-48): one state per text line, in line
 *    order; id, gns and J as strtol(..., 0) (so a leading 0 means octal and
 *    0x hexadecimal, and a field without digits yields 0 and leaves the
 *    cursor where it was), energy as strtod; the state's index is its line
 *    number (the reference indexes states[id - 1] by position).
 *  - .trans (ExomolStateReader.cpp:132-172): per non-empty line, the first
 *    three fields `id_upper id_lower A` as `istream >> int >> int >>
 *    double`; nu = E_upper - E_lower, e_i = E_lower, gns = g_upper.  The
 *    reference reads the file as one token stream, so a line with other
 *    than three fields shifts every later record there; here the fields
 *    after the third are ignored (newer four-column files parse), and a line
 *    with fewer than three fields is an error.
 *  - broadening (ExomolStateReader.cpp:7-37, 39-75): GEXS_BROAD_DEFAULTS
 *    gives every line the default gamma and n, which is what the reference
 *    computes: its lookup key keeps the failed "a1" text after key.clear()
 *    (:21, clear() resets only the stream state), so no "a0" entry ever
 *    matches.  GEXS_BROAD_BY_J applies the intended rule: an "a1" entry for
 *    (J'', J'), else an "a0" entry for J'', else the defaults.
 * Decimal to double conversion is correctly rounded like glibc strtod: an
 * exact fast path for up to 19 significant digits and |exponent| <= 22
 * (one IEEE operation on exact operands), otherwise the digits times 10^k
 * held as a double-double (gen_pow10.py), rounded once; a result can differ
 * from strtod only when the exact value lies within ~2^-100 relative of a
 * rounding midpoint, when it has more than 19 significant digits (the rest
 * are truncated), or when the result is subnormal (below 2.2e-308; it is
 * then rounded twice).  Ingest finally sorts the lines by nu
 * (stable radix sort of the FP64 keys, so equal centres keep file order).
 */
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include "gexs_internal.h"
#include "pow10_dd.h"

namespace gexs {
namespace {

constexpr int64_t CHUNK = 4096;   /* bytes per warp in the newline passes */

/* ------------------------------------------------------------ text index */
__device__ __forceinline__ int count_nl(uint32_t w)
{
    /* bytes equal to '\n' in a 32-bit word */
    const uint32_t x = w ^ 0x0a0a0a0au;
    const uint32_t t = (x - 0x01010101u) & ~x & 0x80808080u;
    return __popc(t);
}

/* newlines in [lane*128, lane*128+128) of the chunk; the chunk start is
 * 16-byte aligned, the tail past n is read byte by byte */
__device__ __forceinline__ int lane_newlines(const uint8_t* text, int64_t n, int64_t base,
                                             int lane)
{
    const int64_t b0 = base + (int64_t)lane * 128;
    int c = 0;
    if (b0 + 128 <= n) {
        const uint4* p = reinterpret_cast<const uint4*>(text + b0);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint4 v = __ldg(p + k);
            c += count_nl(v.x) + count_nl(v.y) + count_nl(v.z) + count_nl(v.w);
        }
    } else {
        for (int64_t i = b0; i < n && i < b0 + 128; ++i) c += (text[i] == '\n');
    }
    return c;
}

__global__ void nl_count_kernel(const uint8_t* __restrict__ text, int64_t n, int64_t nchunk,
                                int64_t* __restrict__ counts)
{
    const int lane = threadIdx.x & 31;
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t ch = w; ch < nchunk; ch += nw) {
        int c = lane_newlines(text, n, ch * CHUNK, lane);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) counts[ch] = c;
    }
}

/* line_end[k] = byte offset of the k-th newline */
__global__ void nl_index_kernel(const uint8_t* __restrict__ text, int64_t n, int64_t nchunk,
                                const int64_t* __restrict__ offsets, int64_t* __restrict__ line_end)
{
    const int lane = threadIdx.x & 31;
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t ch = w; ch < nchunk; ch += nw) {
        const int64_t base = ch * CHUNK;
        const int c = lane_newlines(text, n, base, lane);
        int incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        int64_t k = offsets[ch] + (incl - c);
        const int64_t b0 = base + (int64_t)lane * 128;
        if (c)
            for (int64_t i = b0; i < n && i < b0 + 128; ++i)
                if (text[i] == '\n') line_end[k++] = i;
    }
}

/* --------------------------------------------------------- number parsing */
__device__ __forceinline__ bool is_space(uint8_t c)
{
    return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

/* strtol(p, &next, 0) restricted to [p, end); returns the C long result
 * (clamped on overflow as strtol does) */
__device__ long long strtol0(const uint8_t* p, const uint8_t* end, const uint8_t** next)
{
    const uint8_t* s = p;
    while (s < end && is_space(*s)) ++s;
    bool neg = false;
    if (s < end && (*s == '+' || *s == '-')) { neg = (*s == '-'); ++s; }
    int base = 10;
    auto digit = [&](uint8_t ch) -> int {
        if (ch >= '0' && ch <= '9') return ch - '0';
        if (ch >= 'a' && ch <= 'z') return ch - 'a' + 10;
        if (ch >= 'A' && ch <= 'Z') return ch - 'A' + 10;
        return 99;
    };
    if (s < end && *s == '0') {
        if (s + 2 < end && (s[1] == 'x' || s[1] == 'X') && digit(s[2]) < 16) { base = 16; s += 2; }
        else base = 8;
    }
    const uint8_t* d0 = s;
    unsigned long long v = 0;
    bool ovf = false;
    const unsigned long long lim = neg ? 9223372036854775808ull : 9223372036854775807ull;
    while (s < end) {
        const int dg = digit(*s);
        if (dg >= base) break;
        if (!ovf) {
            if (v > (lim - (unsigned long long)dg) / (unsigned long long)base) ovf = true;
            else v = v * base + dg;
        }
        ++s;
    }
    if (s == d0) { *next = p; return 0; }   /* no conversion: cursor unchanged */
    *next = s;
    if (ovf) return neg ? (-9223372036854775807ll - 1) : 9223372036854775807ll;
    return neg ? -(long long)v : (long long)v;
}

/* istream >> int: whitespace, sign, decimal digits; false if none or the
 * value does not fit an int */
__device__ bool read_int(const uint8_t*& s, const uint8_t* end, int* out)
{
    while (s < end && is_space(*s)) ++s;
    bool neg = false;
    if (s < end && (*s == '+' || *s == '-')) { neg = (*s == '-'); ++s; }
    const uint8_t* d0 = s;
    long long v = 0;
    while (s < end && *s >= '0' && *s <= '9') {
        v = v * 10 + (*s - '0');
        if (v > 2147483648ll) return false;
        ++s;
    }
    if (s == d0) return false;
    if (neg) v = -v;
    if (v > 2147483647ll || v < -2147483648ll) return false;
    *out = (int)v;
    return true;
}

/* M * 10^e correctly rounded (see the file comment), M < 10^19 */
__device__ double scale10(unsigned long long M, int e)
{
    if (M == 0) return 0.0;
    if (M <= (1ull << 53) && e >= -22 && e <= 22) {
        const double m = (double)M;
        const double p = gexs_pow10_dd[e - GEXS_POW10_MIN][0];   /* exact for |e| <= 22 */
        return e >= 0 ? m * p : m / gexs_pow10_dd[-e - GEXS_POW10_MIN][0];
    }
    /* number of digits of M */
    int nd = 1;
    for (unsigned long long t = M; t >= 10; t /= 10) ++nd;
    if (e + nd > 310) return __longlong_as_double(0x7ff0000000000000ll);   /* inf */
    if (e + nd < -343) return 0.0;
    while (e > GEXS_POW10_MAX && M < 1000000000000000000ull) { M *= 10; --e; }
    if (e > GEXS_POW10_MAX) return __longlong_as_double(0x7ff0000000000000ll);
    if (e < GEXS_POW10_MIN) return 0.0;
    /* table entries below 10^GEXS_POW10_SCALED_BELOW carry a factor 2^256:
     * undone by an exact power-of-two scale (rounds twice only for a
     * subnormal result) */
    const double extra = (e < GEXS_POW10_SCALED_BELOW) ? ldexp(1.0, -GEXS_POW10_SCALE_BITS) : 1.0;
    const double mh = (double)M;
    const double ml = (double)(long long)(M - (unsigned long long)mh);
    const double ph = gexs_pow10_dd[e - GEXS_POW10_MIN][0];
    const double pl = gexs_pow10_dd[e - GEXS_POW10_MIN][1];
    /* (mh + ml) * (ph + pl) as hi + lo, rounded once */
    const double hi = mh * ph;
    const double lo = fma(mh, ph, -hi) + (mh * pl + ml * ph);
    return (hi + lo) * extra;
}

/* strtod on [s, end) for decimal input ([sign] digits [. digits] [e [sign]
 * digits]) and inf/infinity/nan; false (cursor unchanged) if no conversion */
__device__ bool read_double(const uint8_t*& s, const uint8_t* end, double* out)
{
    const uint8_t* p = s;
    while (p < end && is_space(*p)) ++p;
    bool neg = false;
    if (p < end && (*p == '+' || *p == '-')) { neg = (*p == '-'); ++p; }
    auto lower = [](uint8_t ch) { return (uint8_t)(ch | 0x20); };
    if (p < end && (lower(*p) == 'i' || lower(*p) == 'n')) {
        if (p + 2 < end && lower(p[0]) == 'i' && lower(p[1]) == 'n' && lower(p[2]) == 'f') {
            p += 3;
            if (p + 4 < end && lower(p[0]) == 'i' && lower(p[1]) == 'n' && lower(p[2]) == 'i' &&
                lower(p[3]) == 't' && lower(p[4]) == 'y') p += 5;
            *out = neg ? -__longlong_as_double(0x7ff0000000000000ll)
                       : __longlong_as_double(0x7ff0000000000000ll);
            s = p;
            return true;
        }
        if (p + 2 < end && lower(p[0]) == 'n' && lower(p[1]) == 'a' && lower(p[2]) == 'n') {
            *out = __longlong_as_double(neg ? (long long)0xfff8000000000000ull : 0x7ff8000000000000ll);
            s = p + 3;
            return true;
        }
        return false;
    }
    /* up to 19 significant digits; later digits are truncated */
    unsigned long long M = 0;
    int nsig = 0, dexp = 0;
    bool any = false;
    while (p < end && *p >= '0' && *p <= '9') {
        any = true;
        if (nsig < 19) { if (M || *p != '0') { M = M * 10 + (*p - '0'); ++nsig; } }
        else ++dexp;
        ++p;
    }
    if (p < end && *p == '.') {
        ++p;
        while (p < end && *p >= '0' && *p <= '9') {
            any = true;
            if (nsig < 19) { if (M || *p != '0') { M = M * 10 + (*p - '0'); ++nsig; } --dexp; }
            ++p;
        }
    }
    if (!any) return false;
    if (p < end && (*p == 'e' || *p == 'E')) {
        const uint8_t* q = p + 1;
        bool eneg = false;
        if (q < end && (*q == '+' || *q == '-')) { eneg = (*q == '-'); ++q; }
        if (q < end && *q >= '0' && *q <= '9') {
            int ev = 0;
            while (q < end && *q >= '0' && *q <= '9') { if (ev < 100000) ev = ev * 10 + (*q - '0'); ++q; }
            dexp += eneg ? -ev : ev;
            p = q;
        }
    }
    const double v = scale10(M, dexp);
    *out = neg ? -v : v;
    s = p;
    return true;
}

/* ----------------------------------------------------------- record parsing */
__device__ __forceinline__ void line_span(const int64_t* __restrict__ line_end, int64_t i,
                                          int64_t nbytes, int64_t* a, int64_t* b)
{
    *a = (i == 0) ? 0 : line_end[i - 1] + 1;
    *b = line_end[i];                 /* the last entry is nbytes for an unterminated tail */
    (void)nbytes;
}

__global__ void states_kernel(const uint8_t* __restrict__ text, int64_t nbytes,
                              const int64_t* __restrict__ line_end, int64_t nlines,
                              double* __restrict__ energy, int32_t* __restrict__ g,
                              int32_t* __restrict__ J, int* __restrict__ err)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nlines;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t a, b;
        line_span(line_end, i, nbytes, &a, &b);
        if (b - a > 1022) { atomicOr(err, 1); continue; }   /* fgets(buffer, 1024) splits it */
        const uint8_t* p = text + a;
        const uint8_t* e = text + b;
        const uint8_t* q;
        (void)strtol0(p, e, &q);                      /* id (unused: states are by position) */
        p = q;
        double en = 0.0;
        const uint8_t* r = p;
        if (read_double(r, e, &en)) p = r;            /* strtod: no conversion keeps p */
        const long long gv = strtol0(p, e, &q);
        p = q;
        const long long jv = strtol0(p, e, &q);
        energy[i] = en;
        g[i] = (int32_t)gv;
        J[i] = (int32_t)jv;
    }
}

__device__ __forceinline__ bool line_has_token(const uint8_t* p, const uint8_t* e)
{
    for (; p < e; ++p) if (!is_space(*p)) return true;
    return false;
}

__global__ void trans_flag_kernel(const uint8_t* __restrict__ text, int64_t nbytes,
                                  const int64_t* __restrict__ line_end, int64_t nlines,
                                  int64_t* __restrict__ flag)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nlines;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t a, b;
        line_span(line_end, i, nbytes, &a, &b);
        flag[i] = line_has_token(text + a, text + b) ? 1 : 0;
    }
}

struct Broad {
    int mode;
    double dgam, dn;
    int n0; const int32_t* j0; const double* g0; const double* x0;    /* a0 by J''      */
    int n1; const int64_t* k1; const double* g1; const double* x1;    /* a1 by (J'', J') */
};

template <typename K>
__device__ __forceinline__ int find_key(const K* keys, int n, K k)
{
    int lo = 0, hi = n;
    while (lo < hi) { const int m = (lo + hi) >> 1; if (keys[m] < k) lo = m + 1; else hi = m; }
    return (lo < n && keys[lo] == k) ? lo : -1;
}

__global__ void trans_kernel(const uint8_t* __restrict__ text, int64_t nbytes,
                             const int64_t* __restrict__ line_end, int64_t nlines,
                             const int64_t* __restrict__ rec, int64_t nstates,
                             const double* __restrict__ sE, const int32_t* __restrict__ sg,
                             const int32_t* __restrict__ sJ, Broad br,
                             double* __restrict__ nu, double* __restrict__ elow,
                             double* __restrict__ aif, int32_t* __restrict__ gns,
                             double* __restrict__ gam, double* __restrict__ nexp,
                             int* __restrict__ err)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nlines;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t a, b;
        line_span(line_end, i, nbytes, &a, &b);
        const uint8_t* p = text + a;
        const uint8_t* e = text + b;
        if (!line_has_token(p, e)) continue;
        const int64_t r = rec[i];
        int idf = 0, idi = 0;
        double A = 0.0;
        if (!read_int(p, e, &idf) || !read_int(p, e, &idi) || !read_double(p, e, &A)) {
            atomicOr(err, 2); continue;
        }
        if (idf < 1 || idi < 1 || idf > nstates || idi > nstates) { atomicOr(err, 4); continue; }
        const int64_t f = idf - 1, l = idi - 1;
        nu[r] = sE[f] - sE[l];
        elow[r] = sE[l];
        aif[r] = A;
        gns[r] = sg[f];
        double gv = br.dgam, nv = br.dn;
        if (br.mode == GEXS_BROAD_BY_J) {
            const int Jl = sJ[l], Ju = sJ[f];
            const int64_t key = ((int64_t)Jl << 32) | (uint32_t)Ju;
            int k = find_key<int64_t>(br.k1, br.n1, key);
            if (k >= 0) { gv = br.g1[k]; nv = br.x1[k]; }
            else if ((k = find_key<int32_t>(br.j0, br.n0, Jl)) >= 0) { gv = br.g0[k]; nv = br.x0[k]; }
        }
        gam[r] = gv;
        nexp[r] = nv;
    }
}

/* ---------------------------------------------------------------- HITRAN
 * 160-column records (Readers/HITRAN/HITRANStateReader.cpp:3-39, 137-250):
 * field widths {2,1,12,10,10,5,5,10,4,8,15,15,15,15,6,12,1,7,7}; a field is
 * read by atof/atoi of its columns (bytes past the end of a short line are
 * absent here; the reference would read stale buffer bytes there). */
__device__ __forceinline__ double field_atof(const uint8_t* a, const uint8_t* b, int off, int len)
{
    const uint8_t* p = a + off;
    const uint8_t* e = (a + off + len < b) ? a + off + len : b;
    double v = 0.0;
    if (p < e) { const uint8_t* q = p; if (!read_double(q, e, &v)) v = 0.0; }
    return v;
}

__global__ void hitran_kernel(const uint8_t* __restrict__ text, int64_t nbytes,
                              const int64_t* __restrict__ line_end, int64_t nlines,
                              const int64_t* __restrict__ rec, double pressure, double mixture,
                              double ref_q,
                              double* __restrict__ nu, double* __restrict__ elow,
                              double* __restrict__ aif, int32_t* __restrict__ gns,
                              double* __restrict__ gam, double* __restrict__ nexp)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nlines;
         i += (int64_t)gridDim.x * blockDim.x) {
        int64_t a, b;
        line_span(line_end, i, nbytes, &a, &b);
        const uint8_t* p = text + a;
        const uint8_t* e = text + b;
        if (!line_has_token(p, e)) continue;
        const int64_t r = rec[i];
        const double v_nu = field_atof(p, e, 3, 12);
        const double v_S = field_atof(p, e, 15, 10);
        double v_A = field_atof(p, e, 25, 10);
        const double g_air = field_atof(p, e, 35, 5);
        const double g_self = field_atof(p, e, 40, 5);
        const double v_E = field_atof(p, e, 45, 10);
        const double v_n = field_atof(p, e, 55, 4);
        double v_g = field_atof(p, e, 146, 7);
        /* (gam_air*mix + self*(1-mix))*P, HITRANStateReader.cpp:218 */
        const double gv = __dmul_rn(__dadd_rn(__dmul_rn(g_air, mixture),
                                              __dmul_rn(g_self, __dsub_rn(1.0, mixture))), pressure);
        if (v_A == 0.0) {
            /* A from S at 296 K and Q(296), :222-247 */
            const double planck = 6.6260693e-27, vellgt = 2.99792458e10, boltz = 1.380658e-16;
            const double pi = 3.141592653589793;
            const double beta = __ddiv_rn(__dmul_rn(planck, vellgt), __dmul_rn(boltz, 296.0));
            double t = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(v_S, 8.0), pi), vellgt), ref_q), v_nu);
            t = __dmul_rn(t, v_nu);
            const double den = __dmul_rn(exp(__dmul_rn(-beta, v_E)), __dsub_rn(1.0, exp(__dmul_rn(-beta, v_nu))));
            v_A = __ddiv_rn(t, den);
            v_g = 1.0;
        }
        nu[r] = v_nu;
        elow[r] = v_E;
        aif[r] = v_A;
        gns[r] = (int32_t)v_g;
        gam[r] = gv;
        nexp[r] = v_n;
    }
}

template <typename T>
__global__ void gather_kernel(const T* __restrict__ in, const int64_t* __restrict__ idx, int64_t n,
                              T* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = in[idx[i]];
}

__global__ void iota_kernel(int64_t* __restrict__ v, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        v[i] = i;
}

/* ------------------------------------------------------------ host helpers */
struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, n ? n : 1); }
    template <typename T> T* as() const { return reinterpret_cast<T*>(p); }
    void* release() { void* q = p; p = nullptr; return q; }
};

int grid_for(gexs_ctx* ctx, int64_t n, int block)
{
    const int nsm = ctx_sm_count(ctx);
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + block - 1) / block, (int64_t)nsm * 16));
}

/* copy text to the device and index its lines: line_end[k] for k < nlines
 * (the last entry is nbytes when the text does not end in a newline) */
int index_text(gexs_ctx* ctx, const char* h_text, int64_t nbytes, DevBuf& d_text,
               DevBuf& d_end, int64_t* nlines, cudaStream_t s)
{
    *nlines = 0;
    if (nbytes == 0) return GEXS_OK;
    if (d_text.alloc((size_t)nbytes + 16) != cudaSuccess) return set_error(GEXS_ERR_OOM, "ingest: text buffer");
    cudaError_t e = cudaMemcpyAsync(d_text.p, h_text, (size_t)nbytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_error(e, "ingest: copy text");
    const int64_t nchunk = (nbytes + CHUNK - 1) / CHUNK;
    /* counts[nchunk] stays 0 so the exclusive scan's last entry is the total */
    DevBuf d_cnt, d_off, d_tmp;
    if (d_cnt.alloc(sizeof(int64_t) * (nchunk + 1)) != cudaSuccess ||
        d_off.alloc(sizeof(int64_t) * (nchunk + 1)) != cudaSuccess)
        return set_error(GEXS_ERR_OOM, "ingest: line index");
    cudaMemsetAsync(d_cnt.p, 0, sizeof(int64_t) * (nchunk + 1), s);
    const int wgrid = grid_for(ctx, nchunk * 32, 256);
    nl_count_kernel<<<wgrid, 256, 0, s>>>(d_text.as<uint8_t>(), nbytes, nchunk, d_cnt.as<int64_t>());
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, d_cnt.as<int64_t>(), d_off.as<int64_t>(), (int)(nchunk + 1), s);
    if (d_tmp.alloc(tb) != cudaSuccess) return set_error(GEXS_ERR_OOM, "ingest: scan");
    cub::DeviceScan::ExclusiveSum(d_tmp.p, tb, d_cnt.as<int64_t>(), d_off.as<int64_t>(), (int)(nchunk + 1), s);
    int64_t nnl = 0;
    e = cudaMemcpyAsync(&nnl, d_off.as<int64_t>() + nchunk, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e, "ingest: count lines");
    char last = 0;
    e = cudaMemcpy(&last, d_text.as<char>() + nbytes - 1, 1, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_error(e, "ingest: last byte");
    const int64_t nl = nnl + (last != '\n' ? 1 : 0);
    if (d_end.alloc(sizeof(int64_t) * (nl + 1)) != cudaSuccess) return set_error(GEXS_ERR_OOM, "ingest: line index");
    nl_index_kernel<<<wgrid, 256, 0, s>>>(d_text.as<uint8_t>(), nbytes, nchunk, d_off.as<int64_t>(),
                                          d_end.as<int64_t>());
    if (last != '\n') {
        const int64_t tail = nbytes;
        cudaMemcpyAsync(d_end.as<int64_t>() + nnl, &tail, sizeof(int64_t), cudaMemcpyHostToDevice, s);
    }
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e, "ingest: index lines");
    *nlines = nl;
    return GEXS_OK;
}

/* stable radix sort of (nu, record) and a gather of every array */
int sort_lines(gexs_ctx* ctx, int64_t nrec, DevBuf& nu, DevBuf& el, DevBuf& A, DevBuf& g,
               DevBuf& gm, DevBuf& nx, cudaStream_t s)
{
    const size_t n8 = sizeof(double) * nrec;
    DevBuf k2, i1, i2, t2;
    if (k2.alloc(n8) != cudaSuccess || i1.alloc(sizeof(int64_t) * nrec) != cudaSuccess ||
        i2.alloc(sizeof(int64_t) * nrec) != cudaSuccess)
        return set_error(GEXS_ERR_OOM, "ingest: sort buffers");
    iota_kernel<<<grid_for(ctx, nrec, 256), 256, 0, s>>>(i1.as<int64_t>(), nrec);
    size_t sb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sb, nu.as<double>(), k2.as<double>(), i1.as<int64_t>(),
                                    i2.as<int64_t>(), nrec, 0, 64, s);
    if (t2.alloc(sb) != cudaSuccess) return set_error(GEXS_ERR_OOM, "ingest: sort");
    cub::DeviceRadixSort::SortPairs(t2.p, sb, nu.as<double>(), k2.as<double>(), i1.as<int64_t>(),
                                    i2.as<int64_t>(), nrec, 0, 64, s);
    const int gg = grid_for(ctx, nrec, 256);
    DevBuf tmp;
    if (tmp.alloc(n8) != cudaSuccess) return set_error(GEXS_ERR_OOM, "ingest: gather");
    auto regather8 = [&](DevBuf& arr) {
        gather_kernel<double><<<gg, 256, 0, s>>>(arr.as<double>(), i2.as<int64_t>(), nrec, tmp.as<double>());
        std::swap(arr.p, tmp.p);
    };
    regather8(el); regather8(A); regather8(gm); regather8(nx);
    gather_kernel<int32_t><<<gg, 256, 0, s>>>(g.as<int32_t>(), i2.as<int64_t>(), nrec, tmp.as<int32_t>());
    std::swap(g.p, tmp.p);
    std::swap(nu.p, k2.p);
    const cudaError_t e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? GEXS_OK : cuda_error(e, "ingest: sort");
}

/* records = non-empty lines, numbered in order: rec[i] for line i, *nrec */
int number_records(gexs_ctx* ctx, const DevBuf& d_text, int64_t nbytes, const DevBuf& d_end,
                   int64_t nl, DevBuf& d_rec, int64_t* nrec, cudaStream_t s)
{
    DevBuf d_flag, d_tmp;
    if (d_flag.alloc(sizeof(int64_t) * (nl + 1)) != cudaSuccess || d_rec.alloc(sizeof(int64_t) * (nl + 1)) != cudaSuccess)
        return set_error(GEXS_ERR_OOM, "ingest: record index");
    cudaMemsetAsync(d_flag.p, 0, sizeof(int64_t) * (nl + 1), s);
    if (nl > 0)
        trans_flag_kernel<<<grid_for(ctx, nl, 256), 256, 0, s>>>(d_text.as<uint8_t>(), nbytes,
                                                                 d_end.as<int64_t>(), nl, d_flag.as<int64_t>());
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, d_flag.as<int64_t>(), d_rec.as<int64_t>(), (int)(nl + 1), s);
    if (d_tmp.alloc(tb) != cudaSuccess) return set_error(GEXS_ERR_OOM, "ingest: scan");
    cub::DeviceScan::ExclusiveSum(d_tmp.p, tb, d_flag.as<int64_t>(), d_rec.as<int64_t>(), (int)(nl + 1), s);
    cudaError_t e = cudaMemcpyAsync(nrec, d_rec.as<int64_t>() + nl, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? GEXS_OK : cuda_error(e, "ingest: count records");
}

/* "code gamma n J'' [J']" lines; codes other than a0/a1 are skipped */
struct BroadHost {
    std::vector<int32_t> j0; std::vector<double> g0, x0;
    std::vector<int64_t> k1; std::vector<double> g1, x1;
};

void parse_broadener(const char* text, int64_t nbytes, BroadHost& bh)
{
    std::vector<std::pair<int32_t, std::pair<double, double>>> a0;
    std::vector<std::pair<int64_t, std::pair<double, double>>> a1;
    int64_t i = 0;
    while (i < nbytes) {
        int64_t j = i;
        while (j < nbytes && text[j] != '\n') ++j;
        std::string line(text + i, text + j);
        i = j + 1;
        char code[16] = {0};
        double g = 0, n = 0;
        int J1 = 0, J2 = 0;
        const int got = std::sscanf(line.c_str(), "%15s %lf %lf %d %d", code, &g, &n, &J1, &J2);
        if (got >= 4 && std::strcmp(code, "a0") == 0) a0.push_back({J1, {g, n}});
        else if (got >= 5 && std::strcmp(code, "a1") == 0)
            a1.push_back({((int64_t)J1 << 32) | (uint32_t)J2, {g, n}});
    }
    /* the first entry of a key wins, as a std::map assignment would keep the last: keep the last */
    auto fin0 = [&]() {
        std::stable_sort(a0.begin(), a0.end(), [](auto& x, auto& y) { return x.first < y.first; });
        for (size_t k = 0; k < a0.size(); ++k) {
            if (k + 1 < a0.size() && a0[k + 1].first == a0[k].first) continue;
            bh.j0.push_back(a0[k].first); bh.g0.push_back(a0[k].second.first); bh.x0.push_back(a0[k].second.second);
        }
    };
    auto fin1 = [&]() {
        std::stable_sort(a1.begin(), a1.end(), [](auto& x, auto& y) { return x.first < y.first; });
        for (size_t k = 0; k < a1.size(); ++k) {
            if (k + 1 < a1.size() && a1[k + 1].first == a1[k].first) continue;
            bh.k1.push_back(a1[k].first); bh.g1.push_back(a1[k].second.first); bh.x1.push_back(a1[k].second.second);
        }
    };
    fin0();
    fin1();
}

int read_file(const char* path, std::vector<char>& buf)
{
    FILE* f = std::fopen(path, "rb");
    if (!f) return set_error(GEXS_ERR_INVALID, std::string("cannot open ") + path);
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf.resize(n > 0 ? (size_t)n : 0);
    const size_t got = n > 0 ? std::fread(buf.data(), 1, (size_t)n, f) : 0;
    std::fclose(f);
    if ((long)got != n) return set_error(GEXS_ERR_INVALID, std::string("short read of ") + path);
    return GEXS_OK;
}

}  // namespace
}  // namespace gexs

using namespace gexs;

extern "C" {

int gexs_exomol_parse_states(gexs_ctx* ctx, const char* h_text, int64_t nbytes,
                             gexs_state_table* out)
{
    if (!ctx || !out || nbytes < 0 || (nbytes > 0 && !h_text))
        return set_error(GEXS_ERR_INVALID, "gexs_exomol_parse_states: arguments");
    std::memset(out, 0, sizeof(*out));
    cudaSetDevice(ctx_device(ctx));
    cudaStream_t s = 0;
    DevBuf d_text, d_end;
    int64_t nl = 0;
    int st = index_text(ctx, h_text, nbytes, d_text, d_end, &nl, s);
    if (st) return st;
    DevBuf dE, dg, dJ, derr;
    if (dE.alloc(sizeof(double) * nl) != cudaSuccess || dg.alloc(sizeof(int32_t) * nl) != cudaSuccess ||
        dJ.alloc(sizeof(int32_t) * nl) != cudaSuccess || derr.alloc(sizeof(int)) != cudaSuccess)
        return set_error(GEXS_ERR_OOM, "gexs_exomol_parse_states: tables");
    cudaMemsetAsync(derr.p, 0, sizeof(int), s);
    if (nl > 0)
        states_kernel<<<grid_for(ctx, nl, 256), 256, 0, s>>>(d_text.as<uint8_t>(), nbytes,
                                                             d_end.as<int64_t>(), nl, dE.as<double>(),
                                                             dg.as<int32_t>(), dJ.as<int32_t>(),
                                                             derr.as<int>());
    int flag = 0;
    cudaError_t e = cudaMemcpyAsync(&flag, derr.p, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e, "gexs_exomol_parse_states");
    if (flag) return set_error(GEXS_ERR_INVALID, "gexs_exomol_parse_states: a line is longer than 1022 bytes");
    out->energy = (double*)dE.release();
    out->g = (int32_t*)dg.release();
    out->J = (int32_t*)dJ.release();
    out->count = nl;
    return GEXS_OK;
}

int gexs_exomol_parse_trans(gexs_ctx* ctx, const gexs_state_table* states, const char* h_text,
                            int64_t nbytes, const char* h_broad, int64_t broad_nbytes,
                            int broad_mode, double default_gamma, double default_n,
                            int sort_by_nu, gexs_line_table* out)
{
    if (!ctx || !states || !out || nbytes < 0 || (nbytes > 0 && !h_text) || broad_nbytes < 0 ||
        (broad_nbytes > 0 && !h_broad) ||
        (broad_mode != GEXS_BROAD_DEFAULTS && broad_mode != GEXS_BROAD_BY_J))
        return set_error(GEXS_ERR_INVALID, "gexs_exomol_parse_trans: arguments");
    std::memset(out, 0, sizeof(*out));
    cudaSetDevice(ctx_device(ctx));
    cudaStream_t s = 0;
    DevBuf d_text, d_end;
    int64_t nl = 0;
    int st = index_text(ctx, h_text, nbytes, d_text, d_end, &nl, s);
    if (st) return st;
    /* records: non-empty lines, numbered in order */
    DevBuf d_flag, d_rec, d_tmp;
    if (d_flag.alloc(sizeof(int64_t) * (nl + 1)) != cudaSuccess || d_rec.alloc(sizeof(int64_t) * (nl + 1)) != cudaSuccess)
        return set_error(GEXS_ERR_OOM, "gexs_exomol_parse_trans: record index");
    cudaMemsetAsync(d_flag.p, 0, sizeof(int64_t) * (nl + 1), s);
    if (nl > 0)
        trans_flag_kernel<<<grid_for(ctx, nl, 256), 256, 0, s>>>(d_text.as<uint8_t>(), nbytes,
                                                                 d_end.as<int64_t>(), nl, d_flag.as<int64_t>());
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, d_flag.as<int64_t>(), d_rec.as<int64_t>(), (int)(nl + 1), s);
    if (d_tmp.alloc(tb) != cudaSuccess) return set_error(GEXS_ERR_OOM, "gexs_exomol_parse_trans: scan");
    cub::DeviceScan::ExclusiveSum(d_tmp.p, tb, d_flag.as<int64_t>(), d_rec.as<int64_t>(), (int)(nl + 1), s);
    int64_t nrec = 0;
    cudaError_t e = cudaMemcpyAsync(&nrec, d_rec.as<int64_t>() + nl, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e, "gexs_exomol_parse_trans: count records");

    /* broadening tables */
    BroadHost bh;
    if (broad_mode == GEXS_BROAD_BY_J && broad_nbytes > 0) parse_broadener(h_broad, broad_nbytes, bh);
    DevBuf dj0, dg0, dx0, dk1, dg1, dx1;
    auto up = [&](DevBuf& d, const void* h, size_t n) -> bool {
        if (d.alloc(n) != cudaSuccess) return false;
        return n == 0 || cudaMemcpyAsync(d.p, h, n, cudaMemcpyHostToDevice, s) == cudaSuccess;
    };
    if (!up(dj0, bh.j0.data(), bh.j0.size() * 4) || !up(dg0, bh.g0.data(), bh.g0.size() * 8) ||
        !up(dx0, bh.x0.data(), bh.x0.size() * 8) || !up(dk1, bh.k1.data(), bh.k1.size() * 8) ||
        !up(dg1, bh.g1.data(), bh.g1.size() * 8) || !up(dx1, bh.x1.data(), bh.x1.size() * 8))
        return set_error(GEXS_ERR_OOM, "gexs_exomol_parse_trans: broadening tables");
    Broad br;
    br.mode = broad_mode; br.dgam = default_gamma; br.dn = default_n;
    br.n0 = (int)bh.j0.size(); br.j0 = dj0.as<int32_t>(); br.g0 = dg0.as<double>(); br.x0 = dx0.as<double>();
    br.n1 = (int)bh.k1.size(); br.k1 = dk1.as<int64_t>(); br.g1 = dg1.as<double>(); br.x1 = dx1.as<double>();

    DevBuf nu, el, A, g, gm, nx, derr;
    const size_t n8 = sizeof(double) * nrec, n4 = sizeof(int32_t) * nrec;
    if (nu.alloc(n8) != cudaSuccess || el.alloc(n8) != cudaSuccess || A.alloc(n8) != cudaSuccess ||
        g.alloc(n4) != cudaSuccess || gm.alloc(n8) != cudaSuccess || nx.alloc(n8) != cudaSuccess ||
        derr.alloc(sizeof(int)) != cudaSuccess)
        return set_error(GEXS_ERR_OOM, "gexs_exomol_parse_trans: line arrays");
    cudaMemsetAsync(derr.p, 0, sizeof(int), s);
    if (nl > 0)
        trans_kernel<<<grid_for(ctx, nl, 256), 256, 0, s>>>(
            d_text.as<uint8_t>(), nbytes, d_end.as<int64_t>(), nl, d_rec.as<int64_t>(), states->count,
            states->energy, states->g, states->J, br, nu.as<double>(), el.as<double>(), A.as<double>(),
            g.as<int32_t>(), gm.as<double>(), nx.as<double>(), derr.as<int>());
    int flag = 0;
    e = cudaMemcpyAsync(&flag, derr.p, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e, "gexs_exomol_parse_trans: parse");
    if (flag & 2) return set_error(GEXS_ERR_INVALID, "gexs_exomol_parse_trans: a line has fewer than three fields");
    if (flag & 4) return set_error(GEXS_ERR_INVALID, "gexs_exomol_parse_trans: state id out of range");

    if (sort_by_nu && nrec > 1) {
        st = sort_lines(ctx, nrec, nu, el, A, g, gm, nx, s);
        if (st) return st;
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "gexs_exomol_parse_trans");
    out->nu = (double*)nu.release(); out->elow = (double*)el.release();
    out->aif = (double*)A.release(); out->gns = (int32_t*)g.release();
    out->gamma = (double*)gm.release(); out->n = (double*)nx.release();
    out->count = nrec;
    return GEXS_OK;
}

int gexs_exomol_load(gexs_ctx* ctx, const char* states_path, const char* trans_path,
                     const char* broad_path, int broad_mode, double default_gamma,
                     double default_n, int sort_by_nu, gexs_state_table* states_out,
                     gexs_line_table* lines_out)
{
    if (!ctx || !states_path || !trans_path || !states_out || !lines_out)
        return set_error(GEXS_ERR_INVALID, "gexs_exomol_load: arguments");
    std::memset(states_out, 0, sizeof(*states_out));
    std::memset(lines_out, 0, sizeof(*lines_out));
    std::vector<char> sbuf, tbuf, bbuf;
    int st = read_file(states_path, sbuf);
    if (st) return st;
    if ((st = read_file(trans_path, tbuf))) return st;
    if (broad_path && broad_path[0]) {
        /* a missing broadener file means defaults, as the reference (:42-46) */
        FILE* f = std::fopen(broad_path, "rb");
        if (f) { std::fclose(f); if ((st = read_file(broad_path, bbuf))) return st; }
    }
    gexs_state_table S;
    st = gexs_exomol_parse_states(ctx, sbuf.data(), (int64_t)sbuf.size(), &S);
    if (st) return st;
    st = gexs_exomol_parse_trans(ctx, &S, tbuf.data(), (int64_t)tbuf.size(), bbuf.data(),
                                 (int64_t)bbuf.size(), broad_mode, default_gamma, default_n,
                                 sort_by_nu, lines_out);
    if (st) { gexs_state_table_free(&S); return st; }
    *states_out = S;
    return GEXS_OK;
}

int gexs_hitran_parse(gexs_ctx* ctx, const char* h_text, int64_t nbytes, double pressure,
                      double air_mixture, double ref_partition_296, int sort_by_nu,
                      gexs_line_table* out)
{
    if (!ctx || !out || nbytes < 0 || (nbytes > 0 && !h_text))
        return set_error(GEXS_ERR_INVALID, "gexs_hitran_parse: arguments");
    std::memset(out, 0, sizeof(*out));
    if (!(ref_partition_296 > 0.0)) {
        /* molecule (columns 1-2) and isotopologue (column 3) of the first
         * record by atoi of their fields (HITRANStateReader.cpp:3-39, 88-95),
         * then TIPS-2011 at 296 K */
        char mol[3] = {0, 0, 0}, iso[2] = {0, 0};
        for (int k = 0; k < 2 && k < nbytes; ++k) mol[k] = h_text[k];
        if (nbytes > 2) iso[0] = h_text[2];
        double gi = 0.0;
        int st = gexs_tips_2011(std::atoi(mol), std::atoi(iso), 296.0, &gi, &ref_partition_296);
        if (st) return st;
    }
    cudaSetDevice(ctx_device(ctx));
    cudaStream_t s = 0;
    DevBuf d_text, d_end, d_rec;
    int64_t nl = 0, nrec = 0;
    int st = index_text(ctx, h_text, nbytes, d_text, d_end, &nl, s);
    if (st) return st;
    if ((st = number_records(ctx, d_text, nbytes, d_end, nl, d_rec, &nrec, s))) return st;
    DevBuf nu, el, A, g, gm, nx;
    const size_t n8 = sizeof(double) * nrec, n4 = sizeof(int32_t) * nrec;
    if (nu.alloc(n8) != cudaSuccess || el.alloc(n8) != cudaSuccess || A.alloc(n8) != cudaSuccess ||
        g.alloc(n4) != cudaSuccess || gm.alloc(n8) != cudaSuccess || nx.alloc(n8) != cudaSuccess)
        return set_error(GEXS_ERR_OOM, "gexs_hitran_parse: line arrays");
    if (nl > 0)
        hitran_kernel<<<grid_for(ctx, nl, 256), 256, 0, s>>>(
            d_text.as<uint8_t>(), nbytes, d_end.as<int64_t>(), nl, d_rec.as<int64_t>(), pressure,
            air_mixture, ref_partition_296, nu.as<double>(), el.as<double>(), A.as<double>(),
            g.as<int32_t>(), gm.as<double>(), nx.as<double>());
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_error(e, "gexs_hitran_parse");
    if (sort_by_nu && nrec > 1 && (st = sort_lines(ctx, nrec, nu, el, A, g, gm, nx, s))) return st;
    out->nu = (double*)nu.release(); out->elow = (double*)el.release();
    out->aif = (double*)A.release(); out->gns = (int32_t*)g.release();
    out->gamma = (double*)gm.release(); out->n = (double*)nx.release();
    out->count = nrec;
    return GEXS_OK;
}

int gexs_state_table_export(const gexs_state_table* t, double* d_energy, int32_t* d_g,
                            int32_t* d_J)
{
    if (!t || (t->count > 0 && (!d_energy || !d_g || !d_J)))
        return set_error(GEXS_ERR_INVALID, "gexs_state_table_export: arguments");
    const size_t n = (size_t)t->count;
    cudaError_t e = cudaMemcpy(d_energy, t->energy, n * sizeof(double), cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_g, t->g, n * sizeof(int32_t), cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_J, t->J, n * sizeof(int32_t), cudaMemcpyDeviceToDevice);
    return e == cudaSuccess ? GEXS_OK : cuda_error(e, "gexs_state_table_export");
}

int gexs_line_table_export(const gexs_line_table* t, double* d_nu, double* d_elow, double* d_aif,
                           int32_t* d_gns, double* d_gamma, double* d_n)
{
    if (!t || (t->count > 0 && (!d_nu || !d_elow || !d_aif || !d_gns || !d_gamma || !d_n)))
        return set_error(GEXS_ERR_INVALID, "gexs_line_table_export: arguments");
    const size_t n8 = (size_t)t->count * sizeof(double), n4 = (size_t)t->count * sizeof(int32_t);
    cudaError_t e = cudaMemcpy(d_nu, t->nu, n8, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_elow, t->elow, n8, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_aif, t->aif, n8, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_gns, t->gns, n4, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_gamma, t->gamma, n8, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_n, t->n, n8, cudaMemcpyDeviceToDevice);
    return e == cudaSuccess ? GEXS_OK : cuda_error(e, "gexs_line_table_export");
}

int gexs_state_table_free(gexs_state_table* t)
{
    if (!t) return GEXS_OK;
    cudaFree(t->energy); cudaFree(t->g); cudaFree(t->J);
    std::memset(t, 0, sizeof(*t));
    return GEXS_OK;
}

int gexs_line_table_free(gexs_line_table* t)
{
    if (!t) return GEXS_OK;
    cudaFree(t->nu); cudaFree(t->elow); cudaFree(t->aif); cudaFree(t->gns);
    cudaFree(t->gamma); cudaFree(t->n);
    std::memset(t, 0, sizeof(*t));
    return GEXS_OK;
}

}  // extern "C"
