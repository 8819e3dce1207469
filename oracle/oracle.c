#define _POSIX_C_SOURCE 200809L
/*
 * oracle.c -- CPU restatement of the GOLAP query hot path, used ONLY as the
 * checker by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.
 * Nothing in the product library links or calls this file.
 *
 * Each function cites the reference code it restates (paths relative to the
 * GOLAP source tree).  Pinning: tests/test_oracle_pin.py checks the SSB
 * generator and the Q1/Q3 restatements against the results of the
 * reference's own code (golden values in tests/golden/), and the LZ4 decoder
 * against liblz4-produced blocks.
 */
#include <stdint.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define OR_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------ LZ4
 * Block-format decoder.  The reference decodes LZ4 on the CPU through
 * LZ4CPUManager::decompress -> LZ4_decompress_safe_partial
 * (core/comp_cpu.hpp:22-27); this restates the published LZ4 block format:
 * sequences of {token, literal-length extension, literals, 16-bit LE offset,
 * match-length extension}, the last sequence being literals only.
 * Returns the decoded size, or -1 on malformed input / overflow. */
OR_EXPORT int64_t or_lz4_decode(const uint8_t* in, uint64_t in_size, uint8_t* out, uint64_t out_cap) {
    uint64_t pos = 0, o = 0;
    for (;;) {
        if (pos >= in_size) return -1;
        uint32_t tok = in[pos++];
        uint64_t lit = tok >> 4;
        if (lit == 15) {
            uint32_t b;
            do {
                if (pos >= in_size) return -1;
                b = in[pos++];
                lit += b;
            } while (b == 255);
        }
        if (pos + lit > in_size || o + lit > out_cap) return -1;
        memcpy(out + o, in + pos, lit);
        o += lit;
        pos += lit;
        if (pos == in_size) return (int64_t)o;
        if (pos + 2 > in_size) return -1;
        uint64_t off = (uint64_t)in[pos] | ((uint64_t)in[pos + 1] << 8);
        pos += 2;
        uint64_t ml = (tok & 15) + 4;
        if ((tok & 15) == 15) {
            uint32_t b;
            do {
                if (pos >= in_size) return -1;
                b = in[pos++];
                ml += b;
            } while (b == 255);
        }
        if (off == 0 || off > o || o + ml > out_cap) return -1;
        for (uint64_t i = 0; i < ml; ++i) out[o + i] = out[o - off + i]; /* byte-serial: overlap-safe */
        o += ml;
    }
}

/* Checks the segment side index of a segmented LZ4 block (own format of the
 * B200 build, no reference counterpart): decodes each segment independently
 * from its entry and compares with the serial decode `ref`.  Returns 0 when
 * every segment reproduces its bytes, else the 1-based failing segment. */
OR_EXPORT int or_lz4_check_segments(const uint8_t* in, uint64_t in_size, const uint32_t* entries, uint32_t S,
                                    uint32_t seg_rows, uint32_t rows, const uint8_t* ref) {
    uint8_t* out = (uint8_t*)malloc((size_t)rows * 4 + 16);
    if (!out) return -2;
    for (uint32_t j = 0; j < S; ++j) {
        uint64_t ob = (uint64_t)(j * seg_rows < rows ? j * seg_rows : rows) * 4;
        uint64_t oe = (uint64_t)((j + 1) * seg_rows < rows ? (j + 1) * seg_rows : rows) * 4;
        uint64_t pos = entries[2 * j], o = ob;
        uint32_t info = entries[2 * j + 1];
        int resume = (info >> 4) & 1;
        uint64_t lit = info >> 5;
        uint32_t mnib = info & 15;
        int bad = 0;
        while (o < oe && !bad) {
            if (!resume) {
                if (pos >= in_size) { bad = 1; break; }
                uint32_t tok = in[pos++];
                lit = tok >> 4;
                mnib = tok & 15;
                if (lit == 15) {
                    uint32_t b;
                    do {
                        if (pos >= in_size) { bad = 1; break; }
                        b = in[pos++];
                        lit += b;
                    } while (b == 255);
                }
            }
            resume = 0;
            uint64_t n = lit < oe - o ? lit : oe - o;
            if (pos + n > in_size) { bad = 1; break; }
            memcpy(out + o, in + pos, n);
            o += n;
            pos += n;
            if (o >= oe) break;
            if (pos + 2 > in_size) { bad = 1; break; }
            uint64_t off = (uint64_t)in[pos] | ((uint64_t)in[pos + 1] << 8);
            pos += 2;
            uint64_t ml = mnib + 4;
            if (mnib == 15) {
                uint32_t b;
                do {
                    if (pos >= in_size) { bad = 1; break; }
                    b = in[pos++];
                    ml += b;
                } while (b == 255);
            }
            /* the segment policy: source inside [ob, o), no crossing of oe */
            if (off == 0 || off > o - ob || o + ml > oe) { bad = 1; break; }
            for (uint64_t i = 0; i < ml; ++i) out[o + i] = out[o - off + i];
            o += ml;
        }
        if (bad || memcmp(out + ob, ref + ob, oe - ob) != 0) {
            free(out);
            return (int)j + 1;
        }
    }
    free(out);
    return 0;
}

/* ------------------------------------------------------------- cascaded
 * Decoder for the build's cascaded block format (RLE + delta + frame of
 * reference bit-packing; layout documented in
 * golap_public_b200/csrc/gx_internal.h).  The reference's cascaded codec is
 * nvCOMP's (core/comp.cuh:237-239), whose stream format is not available;
 * parity for this codec is decode(encode(x)) == x.  Returns rows or -1. */
static uint32_t or_unpack(const uint32_t* w, uint64_t i, uint32_t bits) {
    if (bits == 0) return 0;
    uint64_t bit = i * bits;
    uint64_t two = (uint64_t)w[bit >> 5] | ((uint64_t)w[(bit >> 5) + 1] << 32);
    uint64_t mask = bits == 32 ? 0xFFFFFFFFull : ((1ull << bits) - 1);
    return (uint32_t)((two >> (bit & 31)) & mask);
}

static int64_t or_casc_decode_page(const uint8_t* blk, uint64_t blk_bytes, int32_t* out, uint64_t max_rows) {
    if (blk_bytes < 32) return -1;
    uint32_t h[8];
    memcpy(h, blk, 32);
    uint32_t n_rows = h[0], n_runs = h[1];
    uint32_t flags = h[2] & 255, vbits = (h[2] >> 8) & 255, lbits = (h[2] >> 16) & 255;
    int32_t first = (int32_t)h[3];
    uint32_t vbase = h[4], lbase = h[5], voff = h[6], loff = h[7];
    int rle = flags & 1, delta = (flags >> 1) & 1;
    if (n_rows > max_rows || vbits > 32 || lbits > 32) return -1;
    if (!rle && n_runs != n_rows) return -1;
    if ((uint64_t)voff + 4ull * (((uint64_t)n_runs * vbits + 31) / 32 + 1) > blk_bytes) return -1;
    if (rle && (uint64_t)loff + 4ull * (((uint64_t)n_runs * lbits + 31) / 32 + 1) > blk_bytes) return -1;
    const uint32_t* vw = (const uint32_t*)(blk + voff);
    const uint32_t* lw = (const uint32_t*)(blk + loff);
    uint32_t acc = (uint32_t)first;
    uint64_t r = 0;
    for (uint64_t i = 0; i < n_runs; ++i) {
        uint32_t e = or_unpack(vw, i, vbits) + vbase;
        uint32_t v;
        if (delta) {
            if (i > 0) acc += e;
            v = acc;
        } else {
            v = e;
        }
        uint64_t len = rle ? (uint64_t)or_unpack(lw, i, lbits) + lbase : 1;
        if (r + len > n_rows) return -1;
        for (uint64_t k = 0; k < len; ++k) out[r + k] = (int32_t)v;
        r += len;
    }
    return r == n_rows ? (int64_t)n_rows : -1;
}

/* A cascaded block is a page table {n_pages, page_rows, page_off[n_pages+1]}
 * followed by independently coded pages of page_rows rows (the last one
 * shorter); decodes every page in order.  Returns rows or -1. */
OR_EXPORT int64_t or_casc_decode(const uint8_t* blk, uint64_t blk_bytes, int32_t* out, uint64_t max_rows) {
    if (blk_bytes < 8) return -1;
    uint32_t n_pages, page_rows;
    memcpy(&n_pages, blk, 4);
    memcpy(&page_rows, blk + 4, 4);
    if (page_rows == 0 || (uint64_t)8 + 4ull * ((uint64_t)n_pages + 1) > blk_bytes) return -1;
    uint64_t rows = 0;
    for (uint32_t p = 0; p < n_pages; ++p) {
        uint32_t a, b;
        memcpy(&a, blk + 8 + 4ull * p, 4);
        memcpy(&b, blk + 8 + 4ull * (p + 1), 4);
        if (a > b || b > blk_bytes || (a & 15u)) return -1;
        uint64_t cap = max_rows - rows < page_rows ? max_rows - rows : page_rows;
        int64_t got = or_casc_decode_page(blk + a, b - a, out + rows, cap);
        if (got < 0 || (p + 1 < n_pages && (uint64_t)got != page_rows)) return -1;
        rows += (uint64_t)got;
    }
    return (int64_t)rows;
}

/* ------------------------------------------------------ min/max pruning
 * MinMaxMeta::check_pred_host / check_pred (core/metadata.cuh:195-211):
 * keep a chunk when lo <= chunk_max && hi >= chunk_min (inclusive);
 * MetaChecker::add_minmax ANDs the per-predicate flags
 * (core/metadata.cuh:645-658, combine_and :632-636). */
OR_EXPORT void or_minmax_keep(const int32_t* mins, const int32_t* maxs, uint64_t n, int32_t lo, int32_t hi,
                              uint16_t* keep, int and_into) {
    for (uint64_t c = 0; c < n; ++c) {
        uint16_t k = (lo <= maxs[c] && hi >= mins[c]) ? 1 : 0;
        keep[c] = and_into ? (uint16_t)(keep[c] & k) : k;
    }
}

/* check_mmmeta_multiple_pts (core/metadata.cuh:550-560): keep[c] = 1 where
 * some key lies in [mins[c], maxs[c]] (entries already 1 stay 1). */
OR_EXPORT void or_minmax_points_keep(const int32_t* mins, const int32_t* maxs, uint64_t n, const int32_t* keys,
                                     uint64_t n_keys, uint16_t* keep) {
    for (uint64_t c = 0; c < n; ++c)
        for (uint64_t i = 0; i < n_keys; ++i)
            if (keys[i] >= mins[c] && keys[i] <= maxs[c]) {
                keep[c] = 1;
                break;
            }
}

/* EqHistogram (core/metadata.cuh:225-382): per chunk n_buckets equal-width
 * buckets between the chunk's min and max (add :305-322, double arithmetic),
 * and check_pred (:325-350).  counts has n_chunks * nb entries. */
OR_EXPORT void or_hist_counts(const int32_t* v, uint64_t n, uint64_t rpc, uint32_t nb, const int32_t* mins,
                              const int32_t* maxs, uint64_t* counts) {
    for (uint64_t r = 0; r < n; ++r) {
        const uint64_t c = r / rpc;
        uint64_t b = 0;
        if (maxs[c] != mins[c]) {
            const double inv = (double)nb / (double)((int64_t)maxs[c] - mins[c]);
            b = (uint64_t)((double)((int64_t)v[r] - mins[c]) * inv);
            if (b > nb - 1) b = nb - 1;
        }
        counts[c * nb + b] += 1;
    }
}
OR_EXPORT void or_hist_keep(const int32_t* mins, const int32_t* maxs, const uint64_t* counts, uint64_t n_chunks,
                            uint32_t nb, int32_t lo, int32_t hi, uint16_t* keep) {
    for (uint64_t c = 0; c < n_chunks; ++c) {
        if (mins[c] == maxs[c]) {
            if (lo <= mins[c] && hi >= maxs[c] && counts[c * nb] != 0) keep[c] = 1;
            continue;
        }
        const double inv = (double)nb / (double)((int64_t)maxs[c] - mins[c]);
        int64_t first = (int64_t)(((double)lo - mins[c]) * inv);
        const int64_t last = (int64_t)(((double)hi - mins[c]) * inv);
        if (lo == maxs[c]) first = (int64_t)nb - 1;
        for (int64_t b = 0; b < (int64_t)nb; ++b)
            if (first <= b && last >= b && counts[c * nb + b] != 0) keep[c] = 1;
    }
}

/* BloomMeta (core/metadata.cuh:385-537): (p, m) parameters, the 64-bit
 * finaliser hash (:464-472) and k bits per value per chunk. */
OR_EXPORT uint32_t or_bloom_k(uint64_t m_bytes, double p) {
    const uint64_t mbits = m_bytes << 3;
    const uint64_t nn = (uint64_t)ceil(((double)mbits * log(pow(0.5, log(2.0))) / log(p)));
    return (uint32_t)ceil(log(2.0) * (double)mbits / (double)nn);
}
static uint64_t or_bloom_hash(uint64_t v, uint64_t mbits) {
    v ^= v >> 33;
    v *= 0xff51afd7ed558ccdull;
    v ^= v >> 33;
    v *= 0xc4ceb9fe1a85ec53ull;
    v ^= v >> 33;
    return v % mbits;
}
OR_EXPORT void or_bloom_words(const int32_t* v, uint64_t n, uint64_t rpc, uint64_t m_bytes, uint32_t k,
                              uint32_t* words) {
    const uint64_t mbits = m_bytes << 3, per = m_bytes / 4;
    for (uint64_t r = 0; r < n; ++r) {
        const uint64_t lv = (uint64_t)(int64_t)v[r];
        for (uint32_t i = 0; i < k; ++i) {
            const uint64_t bit = or_bloom_hash(lv + i, mbits);
            words[(r / rpc) * per + (bit >> 5)] |= 1u << (bit & 31);
        }
    }
}
OR_EXPORT void or_bloom_keep(const uint32_t* words, uint64_t n_chunks, uint64_t m_bytes, uint32_t k, int32_t val,
                             uint16_t* keep) {
    const uint64_t mbits = m_bytes << 3, per = m_bytes / 4;
    const uint64_t lv = (uint64_t)(int64_t)val;
    for (uint64_t c = 0; c < n_chunks; ++c) {
        int res = 1;
        for (uint32_t i = 0; i < k; ++i) {
            const uint64_t bit = or_bloom_hash(lv + i, mbits);
            if (!(words[c * per + (bit >> 5)] & (1u << (bit & 31)))) res = 0;
        }
        if (res) keep[c] = 1;
    }
}

/* Per-chunk min/max as collected at ingest by MinMaxMeta::init_chunk
 * (core/metadata.cuh:157-160, CUB min/max reductions). */
OR_EXPORT void or_chunk_minmax(const int32_t* v, uint64_t n, uint64_t rows_per_chunk, int32_t* mins, int32_t* maxs) {
    uint64_t nc = (n + rows_per_chunk - 1) / rows_per_chunk;
    for (uint64_t c = 0; c < nc; ++c) {
        int32_t mn = INT32_MAX, mx = INT32_MIN;
        uint64_t e = (c + 1) * rows_per_chunk < n ? (c + 1) * rows_per_chunk : n;
        for (uint64_t i = c * rows_per_chunk; i < e; ++i) {
            if (v[i] < mn) mn = v[i];
            if (v[i] > mx) mx = v[i];
        }
        mins[c] = mn;
        maxs[c] = mx;
    }
}

/* ------------------------------------------------------------ hash map
 * The reference's chained hash map (HostHashMap, core/host_structs.hpp:10-78;
 * device twin HashMap, core/dev_structs.cuh:37-132): ht_size buckets,
 * hash = key % ht_size, insert pushes rid+1 on the bucket chain, probe walks
 * the chain and returns the first rid whose key matches, else (uint64)-1. */
typedef struct {
    uint64_t ht_size;
    uint64_t* last;   /* bucket heads, rid+1, 0 = empty */
    uint64_t* chain;  /* next pointers per rid */
    const int64_t* keys;
} or_hashmap;

static int or_hm_init(or_hashmap* h, uint64_t ht_size, const int64_t* keys) {
    h->ht_size = ht_size ? ht_size : 1;
    h->keys = keys;
    h->last = (uint64_t*)calloc(h->ht_size, 8);
    h->chain = (uint64_t*)calloc(h->ht_size, 8);
    return h->last && h->chain ? 0 : -1;
}
static void or_hm_free(or_hashmap* h) {
    free(h->last);
    free(h->chain);
}
static void or_hm_insert(or_hashmap* h, uint64_t rid, int64_t key) {
    uint64_t hash = (uint64_t)key % h->ht_size;
    uint64_t prev = h->last[hash];
    h->last[hash] = rid + 1;
    h->chain[rid] = prev;
}
static uint64_t or_hm_probe(const or_hashmap* h, int64_t key) {
    uint64_t hash = (uint64_t)key % h->ht_size;
    for (uint64_t hit = h->last[hash]; hit > 0; hit = h->chain[hit - 1])
        if (h->keys[hit - 1] == key) return hit - 1;
    return (uint64_t)-1;
}

/* Filtered build + probe of a join, returning per probe row the build rid or
 * -1 (hash_map_build_pred_other core/join.cuh:107-135 then
 * HashMap::probe core/dev_structs.cuh:105-113).  build_ok[i] != 0 selects the
 * build rows. */
OR_EXPORT int or_join_probe(const int64_t* build_keys, const uint8_t* build_ok, uint64_t n_build,
                            const int64_t* probe_keys, uint64_t n_probe, int64_t* rid_out) {
    or_hashmap h;
    if (or_hm_init(&h, n_build, build_keys)) return -1;
    for (uint64_t i = 0; i < n_build; ++i)
        if (!build_ok || build_ok[i]) or_hm_insert(&h, i, build_keys[i]);
    for (uint64_t i = 0; i < n_probe; ++i) {
        uint64_t r = or_hm_probe(&h, probe_keys[i]);
        rid_out[i] = r == (uint64_t)-1 ? -1 : (int64_t)r;
    }
    or_hm_free(&h);
    return 0;
}

/* ------------------------------------------------------------------ Q1
 * query1inmem (usecases/ssb/queries/01inmem.hpp:52-141): build the date hash
 * map from the date rows that pass the date predicate (date_ok), then scan
 * the fact rows: discount in [dlo,dhi], quantity in [qlo,qhi], optional
 * extended-price band (:116), probe the date map with the order date, and sum
 * extendedprice*discount into a 64-bit accumulator.  keep_chunk (optional,
 * per rows_per_chunk rows) restricts the scan to surviving chunks, which
 * never changes the result when the flags come from min/max pruning. */
OR_EXPORT int64_t or_q1(const int32_t* lo_orderdate, const int32_t* lo_discount, const int32_t* lo_quantity,
                        const int32_t* lo_extendedprice, uint64_t n, const int32_t* d_key, const uint8_t* date_ok,
                        uint64_t n_date, int32_t dlo, int32_t dhi, int32_t qlo, int32_t qhi, int32_t plo,
                        int32_t phi, const uint16_t* keep_chunk, uint64_t rows_per_chunk) {
    int64_t* keys = (int64_t*)malloc(8 * (n_date ? n_date : 1));
    if (!keys) return INT64_MIN;
    for (uint64_t i = 0; i < n_date; ++i) keys[i] = d_key[i];
    or_hashmap h;
    if (or_hm_init(&h, n_date, keys)) {
        free(keys);
        return INT64_MIN;
    }
    for (uint64_t i = 0; i < n_date; ++i)
        if (date_ok[i]) or_hm_insert(&h, i, keys[i]);
    uint64_t acc = 0;
    for (uint64_t r = 0; r < n; ++r) {
        if (keep_chunk && !keep_chunk[r / rows_per_chunk]) continue;
        if (lo_discount[r] < dlo || lo_discount[r] > dhi || lo_quantity[r] < qlo || lo_quantity[r] > qhi) continue;
        if (lo_extendedprice[r] < plo || lo_extendedprice[r] > phi) continue;
        if (or_hm_probe(&h, lo_orderdate[r]) == (uint64_t)-1) continue;
        acc += (uint64_t)((int64_t)lo_extendedprice[r] * (int64_t)lo_discount[r]);
    }
    or_hm_free(&h);
    free(keys);
    return (int64_t)acc;
}

/* ------------------------------------------------------------------ Q3
 * query3_inmem (usecases/ssb/queries/03inmem.hpp:70-226): three filtered
 * builds (customer, supplier, date), probes in customer -> supplier -> date
 * order with early exit, group {supplier attr, customer attr, date attr}
 * (field order of :176-178), 64-bit revenue sums.  Group keys here are the
 * integer attribute values; results are returned as a dense array
 * sums[((c_attr - c_base) * s_card + (s_attr - s_base)) * d_card + (d_attr - d_base)]
 * plus a per-cell hit count (rows aggregated). */
OR_EXPORT int or_q3(const int32_t* lo_custkey, const int32_t* lo_suppkey, const int32_t* lo_orderdate,
                    const int32_t* lo_revenue, uint64_t n, const int32_t* c_key, const int32_t* c_attr,
                    const uint8_t* c_ok, uint64_t n_c, const int32_t* s_key, const int32_t* s_attr,
                    const uint8_t* s_ok, uint64_t n_s, const int32_t* d_key, const int32_t* d_attr,
                    const uint8_t* d_ok, uint64_t n_d, int32_t c_base, uint32_t c_card, int32_t s_base,
                    uint32_t s_card, int32_t d_base, uint32_t d_card, int64_t* sums, int64_t* counts,
                    const uint16_t* keep_chunk, uint64_t rows_per_chunk) {
    int64_t* kc = (int64_t*)malloc(8 * (n_c ? n_c : 1));
    int64_t* ks = (int64_t*)malloc(8 * (n_s ? n_s : 1));
    int64_t* kd = (int64_t*)malloc(8 * (n_d ? n_d : 1));
    if (!kc || !ks || !kd) return -1;
    for (uint64_t i = 0; i < n_c; ++i) kc[i] = c_key[i];
    for (uint64_t i = 0; i < n_s; ++i) ks[i] = s_key[i];
    for (uint64_t i = 0; i < n_d; ++i) kd[i] = d_key[i];
    or_hashmap hc, hs, hd;
    if (or_hm_init(&hc, n_c, kc) || or_hm_init(&hs, n_s, ks) || or_hm_init(&hd, n_d, kd)) return -1;
    for (uint64_t i = 0; i < n_c; ++i)
        if (c_ok[i]) or_hm_insert(&hc, i, kc[i]);
    for (uint64_t i = 0; i < n_s; ++i)
        if (s_ok[i]) or_hm_insert(&hs, i, ks[i]);
    for (uint64_t i = 0; i < n_d; ++i)
        if (d_ok[i]) or_hm_insert(&hd, i, kd[i]);
    uint64_t cells = (uint64_t)c_card * s_card * d_card;
    memset(sums, 0, 8 * cells);
    memset(counts, 0, 8 * cells);
    int rc = 0;
    for (uint64_t r = 0; r < n; ++r) {
        if (keep_chunk && !keep_chunk[r / rows_per_chunk]) continue;
        uint64_t cm = or_hm_probe(&hc, lo_custkey[r]);
        if (cm == (uint64_t)-1) continue;
        uint64_t sm = or_hm_probe(&hs, lo_suppkey[r]);
        if (sm == (uint64_t)-1) continue;
        uint64_t dm = or_hm_probe(&hd, lo_orderdate[r]);
        if (dm == (uint64_t)-1) continue;
        uint32_t a = (uint32_t)(c_attr[cm] - c_base), b = (uint32_t)(s_attr[sm] - s_base),
                 c = (uint32_t)(d_attr[dm] - d_base);
        if (a >= c_card || b >= s_card || c >= d_card) {
            rc = -2;
            continue;
        }
        uint64_t cell = ((uint64_t)a * s_card + b) * d_card + c;
        sums[cell] += lo_revenue[r];
        counts[cell] += 1;
    }
    or_hm_free(&hc);
    or_hm_free(&hs);
    or_hm_free(&hd);
    free(kc);
    free(ks);
    free(kd);
    return rc;
}

/* --------------------------------------------------------- group by sum
 * HashAggregate::add with SumAgg (core/dev_structs.cuh:210-244,
 * usecases/ssb/queries/query_common.cuh:24-29) as a sort-free CPU sum over a
 * dense key range [0, n_keys). */
/* Q2 shape, the query2 loop (usecases/ssb/queries/02inmem.hpp:100-180):
 * part rows passing part_ok and supplier rows passing supp_ok are joined,
 * every date joins (its year is the group attribute); SUM(revenue) GROUP BY
 * (brand, year) into sums[brand_card][n_years], counts likewise.  Keys are
 * row indexes of the dimension arrays (fact keys index them directly).
 * Returns 0, or -1 on a key outside a dimension. */
OR_EXPORT int or_q2(const int32_t* lo_partkey, const int32_t* lo_suppkey, const int32_t* lo_orderdate,
                    const int32_t* lo_revenue, uint64_t n, const uint8_t* part_ok, const int32_t* p_brand,
                    uint64_t n_part, const uint8_t* supp_ok, uint64_t n_supp, const int32_t* d_key,
                    const int32_t* d_year, uint64_t n_date, int32_t brand_card, int32_t year0, int32_t n_years,
                    int64_t* sums, int64_t* counts) {
    int32_t dmin = INT32_MAX, dmax = INT32_MIN;
    for (uint64_t i = 0; i < n_date; ++i) {
        if (d_key[i] < dmin) dmin = d_key[i];
        if (d_key[i] > dmax) dmax = d_key[i];
    }
    if (n_date == 0) return 0;
    int32_t* dy = (int32_t*)malloc(sizeof(int32_t) * (uint64_t)(dmax - dmin + 1));
    for (int64_t k = 0; k <= (int64_t)dmax - dmin; ++k) dy[k] = INT32_MIN;
    for (uint64_t i = 0; i < n_date; ++i) dy[d_key[i] - dmin] = d_year[i];
    int rc = 0;
    for (uint64_t r = 0; r < n; ++r) {
        const int64_t pk = lo_partkey[r], sk = lo_suppkey[r];
        if (pk < 0 || (uint64_t)pk >= n_part || sk < 0 || (uint64_t)sk >= n_supp) { rc = -1; break; }
        if (!part_ok[pk] || !supp_ok[sk]) continue;
        const int32_t dk = lo_orderdate[r];
        if (dk < dmin || dk > dmax || dy[dk - dmin] == INT32_MIN) continue;
        const int32_t y = dy[dk - dmin] - year0, b = p_brand[pk];
        if (y < 0 || y >= n_years || b < 0 || b >= brand_card) { rc = -1; break; }
        sums[(int64_t)b * n_years + y] += lo_revenue[r];
        counts[(int64_t)b * n_years + y] += 1;
    }
    free(dy);
    return rc;
}

/* Q4 shape, the query4inmem loop (usecases/ssb/queries/04inmem.hpp:120-160):
 * customer / supplier / part rows passing their flags join, dates pass
 * date_ok; SUM(revenue - supplycost) GROUP BY (year, c_nation) into
 * sums[n_years][25], counts likewise. */
OR_EXPORT int or_q4(const int32_t* lo_custkey, const int32_t* lo_suppkey, const int32_t* lo_partkey,
                    const int32_t* lo_orderdate, const int32_t* lo_revenue, const int32_t* lo_supplycost, uint64_t n,
                    const uint8_t* cust_ok, const int32_t* c_nation, uint64_t n_cust, const uint8_t* supp_ok,
                    uint64_t n_supp, const uint8_t* part_ok, uint64_t n_part, const int32_t* d_key,
                    const int32_t* d_year, const uint8_t* date_ok, uint64_t n_date, int32_t year0, int32_t n_years,
                    int64_t* sums, int64_t* counts) {
    int32_t dmin = INT32_MAX, dmax = INT32_MIN;
    for (uint64_t i = 0; i < n_date; ++i) {
        if (d_key[i] < dmin) dmin = d_key[i];
        if (d_key[i] > dmax) dmax = d_key[i];
    }
    if (n_date == 0) return 0;
    int32_t* dy = (int32_t*)malloc(sizeof(int32_t) * (uint64_t)(dmax - dmin + 1));
    for (int64_t k = 0; k <= (int64_t)dmax - dmin; ++k) dy[k] = INT32_MIN;
    for (uint64_t i = 0; i < n_date; ++i)
        if (date_ok[i]) dy[d_key[i] - dmin] = d_year[i];
    int rc = 0;
    for (uint64_t r = 0; r < n; ++r) {
        const int64_t ck = lo_custkey[r], sk = lo_suppkey[r], pk = lo_partkey[r];
        if (ck < 0 || (uint64_t)ck >= n_cust || sk < 0 || (uint64_t)sk >= n_supp || pk < 0 || (uint64_t)pk >= n_part) {
            rc = -1;
            break;
        }
        if (!cust_ok[ck] || !supp_ok[sk] || !part_ok[pk]) continue;
        const int32_t dk = lo_orderdate[r];
        if (dk < dmin || dk > dmax || dy[dk - dmin] == INT32_MIN) continue;
        const int32_t y = dy[dk - dmin] - year0, c = c_nation[ck];
        if (y < 0 || y >= n_years || c < 0 || c >= 25) { rc = -1; break; }
        sums[(int64_t)y * 25 + c] += (int64_t)lo_revenue[r] - lo_supplycost[r];
        counts[(int64_t)y * 25 + c] += 1;
    }
    free(dy);
    return rc;
}

OR_EXPORT int or_group_sum_dense(const int64_t* keys, const int64_t* vals, uint64_t n, int64_t* sums, uint64_t n_keys) {
    memset(sums, 0, 8 * n_keys);
    for (uint64_t i = 0; i < n; ++i) {
        if (keys[i] < 0 || (uint64_t)keys[i] >= n_keys) return -1;
        sums[keys[i]] += vals[i];
    }
    return 0;
}

/* ---------------------------------------------------------- SSB data
 * Restatement of the reference's seeded SSB generator for scale factor sf
 * (usecases/ssb/data/SSB_def.hpp:141-399): LCG uniform_int
 * (core/util.hpp:177-181), table sizes (SSB_def.hpp:147-152), RNG draw order
 * date -> customer -> supplier -> part -> lineorder (:170-176), and the
 * lineorder loop (:201-279).  Only the columns the Q1.x/Q3.x paths read are
 * materialised; all draws are still consumed in the reference order.
 * Nation indices follow the alphabetical order of the NATION map
 * (usecases/ssb/data/SSB_helper.hpp:44-70). */
static uint32_t or_uniform_int(uint64_t* seed, uint32_t a, uint32_t b) {
    *seed = *seed * 1103515245ull + 12345ull;
    return (uint32_t)((((*seed) >> 32) * (uint64_t)(b - a)) >> 32) + a;
}

/* region index of each nation, alphabetical nation order */
static const int32_t OR_NATION_REGION[25] = {0, 1, 1, 1, 2, 4, 0, 3, 3, 2, 2, 4, 4,
                                             2, 4, 0, 0, 0, 1, 3, 3, 4, 3, 1, 2};

typedef struct {
    uint64_t n_lineorder, n_customer, n_supplier, n_part, n_date;
} or_ssb_sizes;

OR_EXPORT void or_ssb_sizes_for(uint32_t sf, uint64_t* n_orders, uint64_t* n_customer, uint64_t* n_supplier,
                                uint64_t* n_part, uint64_t* n_date) {
    uint32_t lg = 0;
    while ((2u << lg) <= sf) ++lg; /* floor(log2(sf)) */
    *n_orders = (uint64_t)sf * 1500000ull;
    *n_part = 200000ull * (uint64_t)(1 + lg);
    *n_supplier = (uint64_t)sf * 2000ull;
    *n_customer = (uint64_t)sf * 30000ull;
    *n_date = 365 * 7;
}

static uint32_t or_partkey_to_price(uint64_t p) {
    uint32_t price = 90000;
    price += (uint32_t)((p / 10) % 20001);
    price += (uint32_t)((p % 1000) * 100);
    return price;
}

/* Fills caller arrays (sized from or_ssb_sizes_for; lineorder arrays need
 * n_orders*7 entries).  Returns the number of lineorder rows. */
/* Part columns are integer codes of the reference strings: p_mfgr
 * "MFGR#m" -> m-1 (0..4), p_category "MFGR#mn" -> 5*(m-1)+(n-1) (0..24),
 * p_brand1 "MFGR#mnbb" -> 40*p_category + (bb-1) (0..999). */
OR_EXPORT int64_t or_ssb_generate(uint32_t sf, uint64_t seed,
                                  /* date */ int32_t* d_key, int32_t* d_year, int32_t* d_yearmonthnum,
                                  int32_t* d_weeknuminyear,
                                  /* customer */ int32_t* c_nation, int32_t* c_region,
                                  /* supplier */ int32_t* s_nation, int32_t* s_region,
                                  /* part (may be NULL) */ int32_t* p_mfgr, int32_t* p_category, int32_t* p_brand1,
                                  /* lineorder */ int32_t* lo_orderdate, int32_t* lo_custkey, int32_t* lo_suppkey,
                                  int32_t* lo_quantity, int32_t* lo_discount, int32_t* lo_extendedprice,
                                  int32_t* lo_revenue, int32_t* lo_partkey, int32_t* lo_supplycost) {
    uint64_t n_orders, n_c, n_s, n_p, n_d;
    or_ssb_sizes_for(sf, &n_orders, &n_c, &n_s, &n_p, &n_d);
    /* populate_date (SSB_def.hpp:372-399): no RNG */
    time_t cur = 694245661;
    for (uint64_t t = 0; t < n_d; ++t) {
        struct tm tmv;
        gmtime_r(&cur, &tmv);
        int y = 1900 + tmv.tm_year;
        d_key[t] = y * 10000 + (tmv.tm_mon + 1) * 100 + tmv.tm_mday;
        d_year[t] = y;
        d_yearmonthnum[t] = y * 100 + tmv.tm_mon + 1;
        d_weeknuminyear[t] = ((tmv.tm_yday + 7 - (tmv.tm_wday ? (tmv.tm_wday - 1) : 6)) / 7) + 1;
        cur += 60 * 60 * 24;
    }
    /* populate_customer (:346-370): nation, city, acode, exchg, pnumber, mktsegment */
    for (uint64_t t = 0; t < n_c; ++t) {
        uint32_t nat = or_uniform_int(&seed, 0, 25);
        for (int k = 0; k < 4; ++k) (void)or_uniform_int(&seed, 0, 10);
        (void)or_uniform_int(&seed, 0, 5);
        c_nation[t] = (int32_t)nat;
        c_region[t] = OR_NATION_REGION[nat];
    }
    /* populate_supplier (:320-344): nation, city, acode, exchg, pnumber */
    for (uint64_t t = 0; t < n_s; ++t) {
        uint32_t nat = or_uniform_int(&seed, 0, 25);
        for (int k = 0; k < 4; ++k) (void)or_uniform_int(&seed, 0, 10);
        s_nation[t] = (int32_t)nat;
        s_region[t] = OR_NATION_REGION[nat];
    }
    /* populate_part (:282-318): size, num1, num2, num3, then 8 draws for the
       type / container / name / colour strings */
    for (uint64_t t = 0; t < n_p; ++t) {
        (void)or_uniform_int(&seed, 1, 51);
        uint32_t num1 = or_uniform_int(&seed, 1, 6), num2 = or_uniform_int(&seed, 1, 6);
        uint32_t num3 = or_uniform_int(&seed, 1, 41);
        for (int k = 0; k < 8; ++k) (void)or_uniform_int(&seed, 0, 10);
        if (p_mfgr) {
            p_mfgr[t] = (int32_t)num1 - 1;
            p_category[t] = 5 * ((int32_t)num1 - 1) + (int32_t)num2 - 1;
            p_brand1[t] = 40 * p_category[t] + (int32_t)num3 - 1;
        }
    }
    /* populate_lineorder (:201-279) */
    uint64_t total = 0;
    for (uint64_t oi = 0; oi < n_orders; ++oi) {
        uint32_t lines = or_uniform_int(&seed, 1, 8);
        int32_t datekey = d_key[or_uniform_int(&seed, 0, (uint32_t)n_d)];
        uint32_t cust;
        do cust = or_uniform_int(&seed, 0, (uint32_t)n_c);
        while (cust % 3 == 0);
        (void)or_uniform_int(&seed, 0, 5); /* priority */
        for (uint32_t li = 0; li < lines; ++li) {
            uint32_t q = or_uniform_int(&seed, 1, 51);
            uint32_t d = or_uniform_int(&seed, 0, 11);
            (void)or_uniform_int(&seed, 0, 9); /* tax */
            uint64_t pk = or_uniform_int(&seed, 0, (uint32_t)n_p);
            uint64_t sk = or_uniform_int(&seed, 0, (uint32_t)n_s);
            uint32_t ext = q * or_partkey_to_price(pk);
            (void)or_uniform_int(&seed, 30, 91); /* commitdate */
            (void)or_uniform_int(&seed, 0, 7);  /* shipmode */
            uint64_t r = total + li;
            lo_orderdate[r] = datekey;
            lo_custkey[r] = (int32_t)cust;
            lo_suppkey[r] = (int32_t)sk;
            lo_quantity[r] = (int32_t)q;
            lo_discount[r] = (int32_t)d;
            lo_extendedprice[r] = (int32_t)ext;
            lo_revenue[r] = (int32_t)(uint32_t)(ext * (100.0 - d) / 100);
            if (lo_partkey) {
                lo_partkey[r] = (int32_t)pk;
                lo_supplycost[r] = (int32_t)(6 * or_partkey_to_price(pk) / 10);
            }
        }
        total += lines;
    }
    return (int64_t)total;
}
