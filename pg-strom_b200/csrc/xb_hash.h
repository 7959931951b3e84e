/*
 * xb_hash.h
 *
 * Hash and numeric helpers shared by host and device code.
 *
 * xb_hash_bytes() is Bob Jenkins' lookup3 "hashlittle" in the form
 * PostgreSQL's hash_any() uses (little-endian word fetch, initial value
 * 0x9e3779b9 + len + 3923095, the final() mix returning c).  PG-Strom's
 * device copy pg_hash_any() (xpu_common.cu:2898-3041) and the host-side
 * inner-relation hash (gpu_join.c:1549-1584 via codegen.c:544-660) must both
 * agree with it, because inner hash tables are built on the host and probed
 * on the device.  The fixed-width variants below are the same function
 * specialised for values already held in registers.
 */
#ifndef XB_HASH_H
#define XB_HASH_H
#include <stdint.h>

#if defined(__CUDACC__)
#define XB_HD __host__ __device__ __forceinline__
#else
#define XB_HD static inline
#endif

#define XB_ROT(x, k)    (((x) << (k)) | ((x) >> (32 - (k))))
#define XB_MIX(a, b, c) do {                        \
        a -= c; a ^= XB_ROT(c, 4);  c += b;          \
        b -= a; b ^= XB_ROT(a, 6);  a += c;          \
        c -= b; c ^= XB_ROT(b, 8);  b += a;          \
        a -= c; a ^= XB_ROT(c, 16); c += b;          \
        b -= a; b ^= XB_ROT(a, 19); a += c;          \
        c -= b; c ^= XB_ROT(b, 4);  b += a;          \
    } while (0)
#define XB_FINAL(a, b, c) do {                      \
        c ^= b; c -= XB_ROT(b, 14);                  \
        a ^= c; a -= XB_ROT(c, 11);                  \
        b ^= a; b -= XB_ROT(a, 25);                  \
        c ^= b; c -= XB_ROT(b, 16);                  \
        a ^= c; a -= XB_ROT(c, 4);                   \
        b ^= a; b -= XB_ROT(a, 14);                  \
        c ^= b; c -= XB_ROT(b, 24);                  \
    } while (0)

/* little-endian gather of up to 4 bytes starting at k[0] */
XB_HD uint32_t xb_le_gather(const uint8_t *k, uint32_t n)
{
    uint32_t v = 0;
    for (uint32_t i = 0; i < n; i++)
        v |= ((uint32_t)k[i]) << (8 * i);
    return v;
}

/* hash_any() over an arbitrary (possibly unaligned) byte string */
XB_HD uint32_t xb_hash_bytes(const uint8_t *k, uint32_t len)
{
    uint32_t a, b, c;
    a = b = c = 0x9e3779b9U + len + 3923095U;
    while (len >= 12) {
        a += xb_le_gather(k, 4);
        b += xb_le_gather(k + 4, 4);
        c += xb_le_gather(k + 8, 4);
        XB_MIX(a, b, c);
        k += 12;
        len -= 12;
    }
    /* the low byte of c is reserved for the length: tail bytes 8..10 go
     * into c shifted up by one byte */
    if (len > 8) {
        c += xb_le_gather(k + 8, len - 8) << 8;
        b += xb_le_gather(k + 4, 4);
        a += xb_le_gather(k, 4);
    } else if (len > 4) {
        b += xb_le_gather(k + 4, len - 4);
        a += xb_le_gather(k, 4);
    } else if (len > 0) {
        a += xb_le_gather(k, len);
    }
    XB_FINAL(a, b, c);
    return c;
}

/* hash_any() of a 1, 2 or 4 byte little-endian value held in a register */
XB_HD uint32_t xb_hash_u32(uint32_t v, uint32_t len)
{
    uint32_t a, b, c;
    a = b = c = 0x9e3779b9U + len + 3923095U;
    if (len < 4)
        v &= (1U << (8 * len)) - 1U;
    a += v;
    XB_FINAL(a, b, c);
    return c;
}

/* hash_any() of an 8 byte value held in a register */
XB_HD uint32_t xb_hash_u64(uint64_t v)
{
    uint32_t a, b, c;
    a = b = c = 0x9e3779b9U + 8U + 3923095U;
    a += (uint32_t)v;
    b += (uint32_t)(v >> 32);
    XB_FINAL(a, b, c);
    return c;
}

/* hash_any() of a 16 byte little-endian int128 (lo, hi) */
XB_HD uint32_t xb_hash_u128(uint64_t lo, uint64_t hi)
{
    uint32_t a, b, c;
    a = b = c = 0x9e3779b9U + 16U + 3923095U;
    a += (uint32_t)lo;
    b += (uint32_t)(lo >> 32);
    c += (uint32_t)hi;
    XB_MIX(a, b, c);
    a += (uint32_t)(hi >> 32);
    XB_FINAL(a, b, c);
    return c;
}

/* pg_hash_merge (xpu_common.h:3470-3476) */
XB_HD uint32_t xb_hash_merge(uint32_t prev, uint32_t next)
{
    return ((prev >> 3) | (prev << 29)) ^ next;
}

/* ----------------------------------------------------------------
 * PostgreSQL numeric varlena -> (kind, scale, int128)
 *
 * Follows __decimal_from_varlena (xpu_numeric.h:216-277): base-10000
 * digits are accumulated into an int128, the scale ("weight" in PG-Strom's
 * naming) is 4 * (ndigits - (pgweight + 1)), then trailing decimal zeros
 * are stripped while the scale is positive (NUMERIC_NORMALIZE).
 * ---------------------------------------------------------------- */
#define XB_NUM_VALID    0
#define XB_NUM_NAN      1
#define XB_NUM_PINF     2
#define XB_NUM_NINF     3

typedef __int128 xb_i128;

/* returns 0 on success, or a non-zero error (1: corrupted, 2: out of range) */
XB_HD int xb_numeric_decode(const uint8_t *vl, uint8_t *p_kind, int16_t *p_weight,
                            xb_i128 *p_value)
{
    uint32_t len, hdr;
    if ((vl[0] & 0x01) == 0x01) {
        if (vl[0] == 0x01)
            return 1;                       /* external toast pointer */
        len = (vl[0] >> 1) & 0x7f;
        hdr = 1;
    } else {
        if ((vl[0] & 0x03) == 0x02)
            return 1;                       /* compressed */
        len = xb_le_gather(vl, 4) >> 2;
        hdr = 4;
    }
    if (len < hdr + 2)
        return 1;
    const uint8_t *nc = vl + hdr;
    uint32_t nc_len = len - hdr;
    uint16_t n_head = (uint16_t)xb_le_gather(nc, 2);
    if ((n_head & 0xC000) == 0xC000) {
        if (n_head == 0xC000)       *p_kind = XB_NUM_NAN;
        else if (n_head == 0xD000)  *p_kind = XB_NUM_PINF;
        else if (n_head == 0xF000)  *p_kind = XB_NUM_NINF;
        else return 1;
        *p_weight = 0;
        *p_value = 0;
        return 0;
    }
    int is_short = ((n_head & 0xC000) == 0x8000);
    int pgweight;
    const uint8_t *digits;
    uint32_t ndigits;
    int negative;
    if (is_short) {
        pgweight = n_head & 0x003F;
        if (n_head & 0x0040)
            pgweight |= ~0x003F;
        digits = nc + 2;
        ndigits = (nc_len - 2) / 2;
        negative = (n_head & 0x2000) != 0;
    } else {
        if (nc_len < 4)
            return 1;
        pgweight = (int16_t)xb_le_gather(nc + 2, 2);
        digits = nc + 4;
        ndigits = (nc_len - 4) / 2;
        negative = (n_head & 0xC000) == 0x4000;
    }
    xb_i128 value = 0;
    for (uint32_t i = 0; i < ndigits; i++) {
        int16_t dig = (int16_t)xb_le_gather(digits + 2 * i, 2);
        if ((value >> 114) != 0)
            return 2;
        value = value * 10000 + dig;
    }
    if (negative)
        value = -value;
    int weight = 4 * ((int)ndigits - (pgweight + 1));
    /* NUMERIC_NORMALIZE */
    if (value == 0) {
        weight = 0;
    } else {
        while (weight > 0) {
            if (weight >= 5 && (value % 100000) == 0) { value /= 100000; weight -= 5; }
            else if (weight >= 4 && (value % 10000) == 0) { value /= 10000; weight -= 4; }
            else if (weight >= 3 && (value % 1000) == 0) { value /= 1000; weight -= 3; }
            else if (weight >= 2 && (value % 100) == 0) { value /= 100; weight -= 2; }
            else if (weight >= 1 && (value % 10) == 0) { value /= 10; weight -= 1; }
            else break;
        }
    }
    *p_kind = XB_NUM_VALID;
    *p_weight = (int16_t)weight;
    *p_value = value;
    return 0;
}

/* rescale an int128 from scale weight_s to weight_d (__normalize_numeric_int128,
 * xpu_numeric.cu:1076-1126: multiply up, or truncate down) */
XB_HD xb_i128 xb_numeric_rescale(int weight_d, int weight_s, xb_i128 v)
{
    int shift;
    if (weight_d > weight_s) {
        for (shift = weight_d - weight_s; shift > 0; ) {
            int k = shift < 18 ? shift : 18;
            xb_i128 p = 1;
            for (int i = 0; i < k; i++) p *= 10;
            v *= p;
            shift -= k;
        }
    } else if (weight_d < weight_s) {
        for (shift = weight_s - weight_d; shift > 0; ) {
            int k = shift < 18 ? shift : 18;
            xb_i128 p = 1;
            for (int i = 0; i < k; i++) p *= 10;
            v /= p;
            shift -= k;
        }
    }
    return v;
}

/* hash of a decoded numeric (xpu_numeric.cu:177-193) */
XB_HD uint32_t xb_hash_numeric(uint8_t kind, int16_t weight, xb_i128 value)
{
    if (kind != XB_NUM_VALID)
        return xb_hash_u32(kind, 1);
    return xb_hash_u32((uint16_t)weight, 2) ^
           xb_hash_u128((uint64_t)value, (uint64_t)(value >> 64));
}

/* order-preserving map of IEEE754 doubles onto int64 (NaN canonicalised as
 * the largest value, as PostgreSQL orders float8) */
XB_HD int64_t xb_f64_ordered(double x)
{
    union { double d; int64_t i; } u;
    u.d = x;
    if (x != x)
        u.i = 0x7ff8000000000000LL;
    return u.i >= 0 ? u.i : (u.i ^ 0x7fffffffffffffffLL);
}
XB_HD double xb_f64_from_ordered(int64_t o)
{
    union { double d; int64_t i; } u;
    u.i = o >= 0 ? o : (o ^ 0x7fffffffffffffffLL);
    return u.d;
}

#endif  /* XB_HASH_H */
