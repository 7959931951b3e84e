/*
 * xb_heapgen.c
 *
 * Seeded-data producer helpers: writes PostgreSQL 8 KB heap pages and
 * MinimalTuple images from column arrays, the way PostgreSQL's
 * heap_fill_tuple / PageAddItem lay them out.  This stands in for the
 * relation files that PG-Strom's relscan.c (pgstromRelScanChunkDirect,
 * relscan.c:555-742) streams into KDS_FORMAT_BLOCK chunks, and for the
 * inner tuples gpu_join.c (execInnerPreloadOneDepth) packs into
 * KDS_FORMAT_HASH; it is test and benchmark infrastructure, not part of
 * the executor.
 *
 * Tuple layout: 23-byte HeapTupleHeader (+ null bitmap when a column is
 * NULL), t_hoff = MAXALIGN(23 + bitmap); fixed-width attributes aligned to
 * attalign; varlena attributes stored as given (1-byte short headers are
 * stored unaligned, 4-byte headers aligned to attalign).
 */
#include <stdint.h>
#include <string.h>

#define BLCKSZ          8192
#define MAXALIGN(x)     (((x) + 7) & ~((int64_t)7))
#define TYPEALIGN(a,x)  (((x) + ((a) - 1)) & ~((int64_t)((a) - 1)))
#define MAX_TUPLES_PER_PAGE 291

typedef struct {
    int32_t attlen;         /* > 0 fixed width, -1 varlena */
    int32_t attalign;       /* 1, 2, 4 or 8 */
} hg_col;

/* size of the data area of row 'r' starting at offset 0 (after t_hoff) */
static int64_t
row_data_size(int ncols, const hg_col *cols, const uint8_t **data,
              const int64_t **voffs, const uint8_t **nulls, int64_t r)
{
    int64_t off = 0;
    for (int j = 0; j < ncols; j++) {
        if (nulls[j] && nulls[j][r])
            continue;
        if (cols[j].attlen > 0) {
            off = TYPEALIGN(cols[j].attalign, off);
            off += cols[j].attlen;
        } else {
            const uint8_t *v = data[j] + voffs[j][r];
            int64_t len = voffs[j][r + 1] - voffs[j][r];
            if (!(v[0] & 0x01))
                off = TYPEALIGN(cols[j].attalign, off);
            off += len;
        }
    }
    return off;
}

static int row_has_null(int ncols, const uint8_t **nulls, int64_t r)
{
    for (int j = 0; j < ncols; j++)
        if (nulls[j] && nulls[j][r])
            return 1;
    return 0;
}

/* writes the data area of row r at 'dst'; returns bytes written */
static int64_t
row_fill(int ncols, const hg_col *cols, const uint8_t **data,
         const int64_t **voffs, const uint8_t **nulls, int64_t r, uint8_t *dst,
         uint8_t *bitmap)
{
    int64_t off = 0;
    for (int j = 0; j < ncols; j++) {
        int isnull = (nulls[j] && nulls[j][r]);
        if (bitmap && !isnull)
            bitmap[j >> 3] |= (uint8_t)(1u << (j & 7));
        if (isnull)
            continue;
        if (cols[j].attlen > 0) {
            int64_t a = TYPEALIGN(cols[j].attalign, off);
            memset(dst + off, 0, a - off);
            off = a;
            memcpy(dst + off, data[j] + (int64_t)cols[j].attlen * r, cols[j].attlen);
            off += cols[j].attlen;
        } else {
            const uint8_t *v = data[j] + voffs[j][r];
            int64_t len = voffs[j][r + 1] - voffs[j][r];
            if (!(v[0] & 0x01)) {
                int64_t a = TYPEALIGN(cols[j].attalign, off);
                memset(dst + off, 0, a - off);
                off = a;
            }
            memcpy(dst + off, v, len);
            off += len;
        }
    }
    return off;
}

/*
 * Fill heap pages with rows [row_begin, nrows).  Pages are written to
 * 'pages' (max_pages * BLCKSZ bytes); block numbers start at first_blkno.
 * Returns the number of pages written; *p_next_row receives the first row
 * that did not fit.
 */
int64_t
hg_build_pages(int ncols, const hg_col *cols, const uint8_t **data,
               const int64_t **voffs, const uint8_t **nulls,
               int64_t row_begin, int64_t nrows,
               uint8_t *pages, int64_t max_pages, uint32_t first_blkno,
               uint32_t xmin, int64_t *p_next_row)
{
    int64_t r = row_begin;
    int64_t np = 0;
    int any_varlena = 0;
    for (int j = 0; j < ncols; j++)
        if (cols[j].attlen < 0)
            any_varlena = 1;
    while (r < nrows && np < max_pages) {
        uint8_t *page = pages + np * BLCKSZ;
        memset(page, 0, BLCKSZ);
        uint32_t lower = 24, upper = BLCKSZ;
        uint32_t nitems = 0;
        while (r < nrows && nitems < MAX_TUPLES_PER_PAGE) {
            int hasnull = row_has_null(ncols, nulls, r);
            int64_t hoff = MAXALIGN(23 + (hasnull ? (ncols + 7) / 8 : 0));
            int64_t len = hoff + row_data_size(ncols, cols, data, voffs, nulls, r);
            int64_t alen = MAXALIGN(len);
            if (lower + 4 > upper - alen)
                break;
            upper -= alen;
            uint8_t *t = page + upper;
            /* HeapTupleHeaderData */
            uint32_t xmax = 0;
            memcpy(t + 0, &xmin, 4);
            memcpy(t + 4, &xmax, 4);
            uint16_t bi_hi = (uint16_t)((first_blkno + np) >> 16);
            uint16_t bi_lo = (uint16_t)((first_blkno + np) & 0xffff);
            uint16_t posid = (uint16_t)(nitems + 1);
            memcpy(t + 12, &bi_hi, 2);
            memcpy(t + 14, &bi_lo, 2);
            memcpy(t + 16, &posid, 2);
            uint16_t infomask2 = (uint16_t)ncols;
            uint16_t infomask = 0x0100 | 0x0200 | 0x0800;   /* frozen, xmax invalid */
            if (hasnull) infomask |= 0x0001;
            if (any_varlena) infomask |= 0x0002;
            memcpy(t + 18, &infomask2, 2);
            memcpy(t + 20, &infomask, 2);
            t[22] = (uint8_t)hoff;
            row_fill(ncols, cols, data, voffs, nulls, r, t + hoff, hasnull ? t + 23 : 0);
            uint32_t lp = (uint32_t)upper | (1u << 15) | ((uint32_t)len << 17);
            memcpy(page + lower, &lp, 4);
            lower += 4;
            nitems++;
            r++;
        }
        if (nitems == 0)
            return -1;      /* a tuple larger than a page */
        /* PageHeaderData */
        uint16_t flags = 0x0004;        /* PD_ALL_VISIBLE */
        uint16_t lo16 = (uint16_t)lower, up16 = (uint16_t)upper, sp16 = BLCKSZ;
        uint16_t ver = BLCKSZ | 4;
        memcpy(page + 10, &flags, 2);
        memcpy(page + 12, &lo16, 2);
        memcpy(page + 14, &up16, 2);
        memcpy(page + 16, &sp16, 2);
        memcpy(page + 18, &ver, 2);
        np++;
    }
    *p_next_row = r;
    return np;
}

/*
 * Size in bytes of the MinimalTuple image of row r (t_len), as stored in a
 * KDS_FORMAT_HASH inner buffer before the trailing row-id.
 */
int64_t
hg_minimal_tuple_len(int ncols, const hg_col *cols, const uint8_t **data,
                     const int64_t **voffs, const uint8_t **nulls, int64_t r)
{
    int hasnull = row_has_null(ncols, nulls, r);
    int64_t hoff = MAXALIGN(23 + (hasnull ? (ncols + 7) / 8 : 0));
    return hoff - 8 + row_data_size(ncols, cols, data, voffs, nulls, r);
}

/*
 * Write the KDS_FORMAT_HASH body for rows [0, nrows): hash slots (chains by
 * hash % nslots, most recent first), row index and kern_hashitem images at
 * the tail, laid out as __innerPreloadSetupHashBuffer does
 * (gpu_join.c:2129-2164).  'kds' points at the KDS base; head_len is its
 * header length; the KDS length must already be set to kds_length.
 */
int64_t
hg_build_hash_kds(int ncols, const hg_col *cols, const uint8_t **data,
                  const int64_t **voffs, const uint8_t **nulls, int64_t nrows,
                  const uint32_t *hashes, uint8_t *kds, int64_t head_len,
                  uint32_t nslots, int64_t kds_length)
{
    uint64_t *hslot = (uint64_t *)(kds + head_len);
    uint64_t *rowindex = hslot + nslots;
    uint8_t *tail = kds + kds_length;
    uint8_t *cur = tail;
    int any_varlena = 0;
    for (int j = 0; j < ncols; j++)
        if (cols[j].attlen < 0)
            any_varlena = 1;
    for (int64_t r = 0; r < nrows; r++) {
        int hasnull = row_has_null(ncols, nulls, r);
        int64_t hoff = MAXALIGN(23 + (hasnull ? (ncols + 7) / 8 : 0));
        int64_t t_len = hoff - 8 + row_data_size(ncols, cols, data, voffs, nulls, r);
        int64_t isz = MAXALIGN(8 + t_len + 4);
        cur -= isz;
        if ((uint8_t *)(rowindex + nrows) > cur)
            return -1;
        memset(cur, 0, isz);
        uint64_t self = (uint64_t)(tail - cur);
        uint32_t hidx = hashes[r] % nslots;
        uint64_t next = hslot[hidx];
        hslot[hidx] = self;
        memcpy(cur, &next, 8);
        uint8_t *t = cur + 8;                       /* kern_tupitem */
        uint32_t tl = (uint32_t)(t_len + 4);
        memcpy(t + 0, &tl, 4);
        memcpy(t + 4, &hashes[r], 4);
        uint16_t infomask2 = (uint16_t)ncols;
        uint16_t infomask = (hasnull ? 0x0001 : 0) | (any_varlena ? 0x0002 : 0);
        memcpy(t + 10, &infomask2, 2);
        memcpy(t + 12, &infomask, 2);
        t[14] = (uint8_t)hoff;                      /* heap t_hoff (incl. 8-byte offset) */
        row_fill(ncols, cols, data, voffs, nulls, r, t + hoff - 8, hasnull ? t + 15 : 0);
        uint32_t rowid = (uint32_t)r;
        memcpy(t + tl - 4, &rowid, 4);
        rowindex[r] = (uint64_t)(tail - t);
    }
    return (int64_t)(tail - cur);
}
