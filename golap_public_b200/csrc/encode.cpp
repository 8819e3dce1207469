// encode.cpp -- host-side column ingest: chunking, per-block LZ4 / cascaded
// encoding and per-chunk min/max collection.
//
// Counterpart of the reference ingest path prepare_compressed
// (core/apps.cuh:149-255), which runs nvCOMP's ChunkCompressor per chunk
// (core/comp.cuh:81-148) and then MinMaxMeta::init_chunk
// (core/metadata.cuh:157-160).  Here one pass over the host column produces
// the compressed blocks, the block directory (BlockInfo, core/comp.cuh:23-32)
// and the chunk min/max; blocks are encoded in parallel host threads.
#include <algorithm>
#include <cstring>
#include <atomic>
#include <thread>

#include "gx_internal.h"
#include "../../include/gx.h"

namespace gx {
namespace {

inline uint32_t bits_for(uint64_t range) {
    return range == 0 ? 0u : (uint32_t)(64 - __builtin_clzll(range));
}

inline void put_u8(std::vector<uint8_t>& o, uint8_t v) { o.push_back(v); }

inline void put_len_ext(std::vector<uint8_t>& o, uint32_t rem) {
    // LZ4 length extension: 255-bytes until the remainder is < 255.
    while (rem >= 255) {
        o.push_back(255);
        rem -= 255;
    }
    o.push_back((uint8_t)rem);
}

inline uint32_t ext_bytes(uint32_t len) {  // extension bytes for a 4-bit field holding len
    return len >= 15 ? (len - 15) / 255 + 1 : 0;
}

struct SeqEmitter {
    std::vector<uint8_t>& out;
    uint32_t n_seq = 0;     // sequences emitted
    size_t base;            // offset of the block start in out
    const uint8_t* bytes;   // input block as bytes
    uint32_t* seg;          // 2*S entries
    const uint32_t* bound;  // boundary word positions, S+1 entries
    uint32_t S;
    uint32_t next_b = 1;    // next unresolved boundary (entry 0 is fixed)

    // Emit literals [anchor, m) and, if has_match, a match of mlen words at
    // offset off words.  Resolves segment entries whose boundary lies in
    // [anchor, m] (or [anchor, end) for the final literal-only sequence).
    void emit(uint32_t anchor, uint32_t m, bool has_match, uint32_t off_w, uint32_t mlen_w) {
        ++n_seq;
        const uint32_t tp = (uint32_t)(out.size() - base);
        const uint32_t Lb = (m - anchor) * 4;
        const uint32_t Mb = mlen_w * 4;
        const uint32_t mnib = has_match ? std::min<uint32_t>(Mb - 4, 15) : 0;
        const uint32_t lit0 = tp + 1 + ext_bytes(Lb);
        if (n_seq == 1 && Lb > 0) {
            // entry 0 resumes inside the block's first literal run (not at its token),
            // so a tile at the block start whose rows are literals is a plain byte range
            seg[0] = lit0;
            seg[1] = (Lb << 5) | 16u | mnib;
        }
        while (next_b < S) {
            uint32_t N = bound[next_b];
            if (N == anchor) {
                seg[2 * next_b] = tp;
                seg[2 * next_b + 1] = 0;
            } else if (N > anchor && (has_match ? N <= m : N < m)) {
                seg[2 * next_b] = lit0 + (N - anchor) * 4;
                seg[2 * next_b + 1] = (((m - N) * 4) << 5) | 16u | mnib;
            } else {
                break;
            }
            ++next_b;
        }
        put_u8(out, (uint8_t)((std::min<uint32_t>(Lb, 15) << 4) | mnib));
        if (Lb >= 15) put_len_ext(out, Lb - 15);
        out.insert(out.end(), bytes + anchor * 4, bytes + m * 4);
        if (has_match) {
            uint32_t off = off_w * 4;
            put_u8(out, (uint8_t)(off & 255));
            put_u8(out, (uint8_t)(off >> 8));
            if (Mb - 4 >= 15) put_len_ext(out, Mb - 4 - 15);
        }
    }
    // Boundaries at the very end of the block (empty trailing segments).
    void finish(uint32_t end_pos) {
        const uint32_t comp_end = (uint32_t)(out.size() - base);
        while (next_b < S) {
            seg[2 * next_b] = comp_end;
            seg[2 * next_b + 1] = 16u;
            (void)end_pos;
            ++next_b;
        }
    }
};

}  // namespace

// Word-granular LZ4 block encoder with the segment policy described in
// gx_internal.h.  Greedy longest match over a hash chain restricted to the
// current segment.
size_t lz4_encode_block(const int32_t* vals, uint32_t W, uint32_t S, uint32_t seg_rows,
                        uint32_t min_match, uint32_t depth, std::vector<uint8_t>& out,
                        uint32_t* seg, uint32_t* n_seq) {
    constexpr uint32_t HB = 14;
    const size_t base = out.size();
    std::vector<uint32_t> bound(S + 1);
    for (uint32_t j = 0; j <= S; ++j) bound[j] = std::min<uint64_t>((uint64_t)j * seg_rows, W);
    seg[0] = 0;
    seg[1] = 0;
    SeqEmitter em{out, 0, base, (const uint8_t*)vals, seg, bound.data(), S};
    const uint32_t min_w = std::max<uint32_t>(1, (min_match + 3) / 4);
    if (min_w >= W) {  // no match can be long enough: the block is one literal run
        em.emit(0, W, false, 0, 0);
        em.finish(W);
        if (n_seq) *n_seq = em.n_seq;
        return out.size() - base;
    }
    std::vector<int32_t> head(1u << HB, -1);
    std::vector<int32_t> prev(W ? W : 1, -1);
    const uint32_t* v = (const uint32_t*)vals;
    auto h = [&](uint32_t x) { return (x * 2654435761u) >> (32 - HB); };
    uint32_t anchor = 0;
    for (uint32_t j = 0; j < S; ++j) {
        const uint32_t a = bound[j], b = bound[j + 1];
        uint32_t p = a;
        const uint32_t lim = std::min<uint32_t>(b, W >= 2 ? W - 2 : 0);  // match end limit
        while (p < b) {
            uint32_t best_len = 0, best_q = 0;
            if (W >= 3 && p + 3 <= W && p < lim) {
                int32_t q = head[h(v[p])];
                uint32_t d = 0;
                while (q >= (int32_t)a && d < depth) {
                    if (v[q] == v[p]) {
                        uint32_t len = 1;
                        while (p + len < lim && v[q + len] == v[p + len]) ++len;
                        if (len > best_len) {
                            best_len = len;
                            best_q = (uint32_t)q;
                        }
                    }
                    q = prev[q];
                    ++d;
                }
            }
            if (best_len >= min_w) {
                em.emit(anchor, p, true, p - best_q, best_len);
                for (uint32_t k = 0; k < best_len; ++k) {
                    uint32_t hk = h(v[p + k]);
                    prev[p + k] = head[hk];
                    head[hk] = (int32_t)(p + k);
                }
                p += best_len;
                anchor = p;
            } else {
                uint32_t hk = h(v[p]);
                prev[p] = head[hk];
                head[hk] = (int32_t)p;
                ++p;
            }
        }
    }
    em.emit(anchor, W, false, 0, 0);
    em.finish(W);
    if (n_seq) *n_seq = em.n_seq;
    return out.size() - base;
}

// Decode-cost-aware policy (lz4_min_match = 0): the block is encoded with
// minimum matches of 1, 2 and 4 words and with no matches at all, and the
// encoding with the lowest bytes + kSeqCost * sequences (+ kMatchCost when it
// has any match) is kept.  A sequence costs the GPU decoder a serial header
// parse, worth about kSeqCost bytes of streaming, and a block of literals
// only decodes as a flat copy, several times faster than parsing: short
// matches that save a byte or two each are not worth it, long matches (runs,
// repeated stretches) are.
size_t lz4_encode_block_auto(const int32_t* vals, uint32_t W, uint32_t S, uint32_t seg_rows, uint32_t depth,
                             std::vector<uint8_t>& out, uint32_t* seg) {
    constexpr uint64_t kSeqCost = 24, kMatchCost = 2048;
    const uint32_t cands[4] = {4, 8, 16, 0xFFFFFFF0u};  // the last admits no match
    std::vector<uint8_t> best_buf, tmp;
    std::vector<uint32_t> best_seg(2 * (size_t)S), tmp_seg(2 * (size_t)S);
    uint64_t best_cost = UINT64_MAX;
    for (uint32_t mm : cands) {
        tmp.clear();
        uint32_t ns = 0;
        const size_t used = lz4_encode_block(vals, W, S, seg_rows, mm, depth, tmp, tmp_seg.data(), &ns);
        const uint64_t cost = used + kSeqCost * ns + (ns > 1 ? kMatchCost : 0);
        if (cost < best_cost) {
            best_cost = cost;
            best_buf.swap(tmp);
            best_seg.swap(tmp_seg);
        }
    }
    out.insert(out.end(), best_buf.begin(), best_buf.end());
    std::memcpy(seg, best_seg.data(), 8ull * S);
    return best_buf.size();
}

// One cascaded page (at most kCascPageRows rows): the smallest of
// {plain, delta} x {no RLE, RLE with at most kCascPageMaxRuns runs}.
size_t casc_encode_page(const int32_t* vals, uint32_t rows, bool allow_rle, bool allow_delta,
                        bool allow_bp, std::vector<uint8_t>& out) {
    // runs
    std::vector<int32_t> rv;
    std::vector<uint32_t> rl;
    if (allow_rle) {
        for (uint32_t i = 0; i < rows;) {
            uint32_t k = i + 1;
            while (k < rows && vals[k] == vals[i]) ++k;
            rv.push_back(vals[i]);
            rl.push_back(k - i);
            i = k;
            if (rv.size() > kCascPageMaxRuns) break;
        }
    }
    const bool rle_ok = allow_rle && rv.size() <= kCascPageMaxRuns && rows > 0;
    struct Cand {
        bool rle, delta;
        uint32_t n, vbits, lbits;
        int64_t vbase;
        uint32_t lbase;
        size_t bytes;
    };
    auto words_for = [](uint64_t n, uint32_t w) -> size_t {
        return (size_t)((n * w + 31) / 32) + 1;  // + 1 padding word
    };
    auto a16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    auto evaluate = [&](bool rle, bool delta) {
        Cand c{rle, delta, 0, 0, 0, 0, 0, 0};
        const int32_t* src = rle ? rv.data() : vals;
        c.n = rle ? (uint32_t)rv.size() : rows;
        int64_t mn = INT64_MAX, mx = INT64_MIN;
        for (uint32_t i = 0; i < c.n; ++i) {
            int64_t e = delta ? (i == 0 ? 0 : (int64_t)(int32_t)((uint32_t)src[i] - (uint32_t)src[i - 1]))
                              : (int64_t)src[i];
            mn = std::min(mn, e);
            mx = std::max(mx, e);
        }
        if (c.n == 0) mn = mx = 0;
        if (allow_bp) {
            c.vbase = mn;
            c.vbits = bits_for((uint64_t)(mx - mn));
        } else {
            c.vbase = 0;
            c.vbits = 32;
        }
        c.bytes = 32 + a16(4 * words_for(c.n, c.vbits));
        if (rle) {
            uint32_t lmn = UINT32_MAX, lmx = 0;
            for (uint32_t x : rl) {
                lmn = std::min(lmn, x);
                lmx = std::max(lmx, x);
            }
            if (allow_bp) {
                c.lbase = lmn;
                c.lbits = bits_for(lmx - lmn);
            } else {
                c.lbase = 0;
                c.lbits = 32;
            }
            c.bytes += a16(4 * words_for(c.n, c.lbits));
        }
        return c;
    };
    Cand best = evaluate(false, false);
    auto consider = [&](bool rle, bool delta) {
        Cand c = evaluate(rle, delta);
        if (c.bytes < best.bytes) best = c;
    };
    if (allow_delta) consider(false, true);
    if (rle_ok) {
        consider(true, false);
        if (allow_delta) consider(true, true);
    }
    // write
    const size_t base = out.size();
    out.resize(base + best.bytes, 0);
    uint8_t* blk = out.data() + base;
    casc_hdr hd{};
    hd.n_rows = rows;
    hd.n_runs = best.n;
    hd.flags = (uint8_t)((best.rle ? CASC_RLE : 0) | (best.delta ? CASC_DELTA : 0));
    hd.val_bits = (uint8_t)best.vbits;
    hd.len_bits = (uint8_t)(best.rle ? best.lbits : 0);
    const int32_t* src = best.rle ? rv.data() : vals;
    hd.first = best.n ? src[0] : 0;
    hd.val_base = (int32_t)(uint32_t)(uint64_t)best.vbase;
    hd.len_base = best.rle ? best.lbase : 0;
    hd.vals_off = 32;
    size_t vbytes = a16(4 * words_for(best.n, best.vbits));
    hd.lens_off = best.rle ? (uint32_t)(32 + vbytes) : 0;
    std::memcpy(blk, &hd, sizeof(hd));
    auto pack = [](uint32_t* words, uint32_t i, uint32_t w, uint32_t u) {
        if (w == 0) return;
        uint64_t bit = (uint64_t)i * w;
        uint32_t wi = (uint32_t)(bit >> 5), sh = (uint32_t)(bit & 31);
        words[wi] |= u << sh;
        if (sh + w > 32) words[wi + 1] |= (uint32_t)((uint64_t)u >> (32 - sh));
    };
    uint32_t* vw = (uint32_t*)(blk + hd.vals_off);
    for (uint32_t i = 0; i < best.n; ++i) {
        int64_t e = best.delta ? (i == 0 ? 0 : (int64_t)(int32_t)((uint32_t)src[i] - (uint32_t)src[i - 1]))
                               : (int64_t)src[i];
        pack(vw, i, best.vbits, (uint32_t)(uint64_t)(e - best.vbase));
    }
    if (best.rle) {
        uint32_t* lw = (uint32_t*)(blk + hd.lens_off);
        for (uint32_t i = 0; i < best.n; ++i) pack(lw, i, best.lbits, rl[i] - best.lbase);
    }
    return best.bytes;
}

// A cascaded block: the page table, then one page per kCascPageRows rows
// (format in gx_internal.h).  page_entries receives {page_off, page_bytes}
// per page (the column's side index).
size_t casc_encode_block(const int32_t* vals, uint32_t rows, bool allow_rle, bool allow_delta,
                         bool allow_bp, std::vector<uint8_t>& out, uint32_t* page_entries) {
    const size_t base = out.size();
    const uint32_t n_pages = (rows + kCascPageRows - 1) / kCascPageRows;
    const size_t hdr = (8 + 4 * ((size_t)n_pages + 1) + 15) & ~(size_t)15;
    out.resize(base + hdr, 0);
    std::vector<uint32_t> off(n_pages + 1);
    for (uint32_t p = 0; p < n_pages; ++p) {
        off[p] = (uint32_t)(out.size() - base);
        const uint32_t r0 = p * kCascPageRows;
        casc_encode_page(vals + r0, std::min(kCascPageRows, rows - r0), allow_rle, allow_delta, allow_bp, out);
        out.resize((out.size() + 15) & ~(size_t)15, 0);  // pages start 16-byte aligned
        page_entries[2 * p] = off[p];
        page_entries[2 * p + 1] = (uint32_t)(out.size() - base) - off[p];
    }
    off[n_pages] = (uint32_t)(out.size() - base);
    uint32_t* h = (uint32_t*)(out.data() + base);
    h[0] = n_pages;
    h[1] = kCascPageRows;
    std::memcpy(h + 2, off.data(), 4ull * (n_pages + 1));
    return out.size() - base;
}

// Offset of the first literal byte of an LZ4 block that opens with literals
// (token, then the literal-length extension), or -1.
static long lz4_first_literal(const uint8_t* blk, size_t n) {
    if (n == 0 || (blk[0] >> 4) == 0) return -1;
    size_t p = 1;
    if ((blk[0] >> 4) == 15) {
        while (p < n && blk[p] == 255) ++p;
        ++p;
    }
    return p <= n ? (long)p : -1;
}

int column_encode(const int32_t* vals, uint64_t n_rows, uint32_t codec, uint32_t rows_per_chunk,
                  uint32_t rows_per_block, uint32_t S, uint32_t min_match, uint32_t depth,
                  bool rle, bool delta, bool bp, uint32_t threads, gx_column* col) {
    if (n_rows == 0) return set_error(GX_ERR_INVALID, "column_encode: empty column");
    if (rows_per_block == 0 || rows_per_block > kMaxRowsPerBlock)
        return set_error(GX_ERR_INVALID, "rows_per_block must be in 1..%u", kMaxRowsPerBlock);
    if (rows_per_chunk == 0) return set_error(GX_ERR_INVALID, "rows_per_chunk must be > 0");
    if (codec > GX_CODEC_CASCADED) return set_error(GX_ERR_INVALID, "unknown codec %u", codec);
    if (codec == GX_CODEC_LZ4) {
        if (S == 0 || S > kMaxSegments || (S & (S - 1)) != 0)
            return set_error(GX_ERR_INVALID, "lz4_segments must be a power of two in 1..%u", kMaxSegments);
        if (S > 1 && ((rows_per_block & (rows_per_block - 1)) != 0 || rows_per_block < S))
            return set_error(GX_ERR_INVALID, "segmented LZ4 needs a power-of-two rows_per_block >= segments");
        if (min_match != 0 && (min_match < 4 || (min_match & 3)))
            return set_error(GX_ERR_INVALID, "lz4_min_match must be 0 (decode-cost-aware) or a multiple of 4 >= 4");
    } else if (codec == GX_CODEC_CASCADED) {
        S = (rows_per_block + kCascPageRows - 1) / kCascPageRows;  // pages per block
    } else {
        S = 1;
    }
    col->n_rows = n_rows;
    col->codec = codec;
    col->rows_per_chunk = rows_per_chunk;
    col->rows_per_block = rows_per_block;
    col->n_chunks = (uint32_t)((n_rows + rows_per_chunk - 1) / rows_per_chunk);
    col->blocks_per_chunk = (rows_per_chunk + rows_per_block - 1) / rows_per_block;
    col->n_slots = col->n_chunks * col->blocks_per_chunk;
    col->S = S;
    col->seg_shift = 0;
    if (codec == GX_CODEC_CASCADED) {
        col->seg_shift = kCascPageLog2;
    } else if (S > 1) {
        uint32_t sr = rows_per_block / S;
        while ((1u << col->seg_shift) < sr) ++col->seg_shift;
    }
    col->blocks.assign(col->n_slots, gx_dblock{0, 0, 0});
    if (S > 1 || codec == GX_CODEC_CASCADED) col->seg.assign((size_t)2 * S * col->n_slots, 0);
    col->mins.assign(col->n_chunks, 0);
    col->maxs.assign(col->n_chunks, 0);
    col->bmins.assign(col->n_slots, INT32_MAX);  // absent slots keep the empty range
    col->bmaxs.assign(col->n_slots, INT32_MIN);

    // min/max per chunk (inclusive)
    for (uint32_t c = 0; c < col->n_chunks; ++c) {
        uint64_t r0 = (uint64_t)c * rows_per_chunk;
        uint64_t r1 = std::min<uint64_t>(n_rows, r0 + rows_per_chunk);
        int32_t mn = INT32_MAX, mx = INT32_MIN;
        for (uint64_t r = r0; r < r1; ++r) {
            mn = std::min(mn, vals[r]);
            mx = std::max(mx, vals[r]);
        }
        col->mins[c] = mn;
        col->maxs[c] = mx;
    }

    // parallel block encoding into per-thread buffers
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    threads = std::min<uint32_t>(threads, std::max<uint32_t>(1, col->n_slots));
    std::vector<std::vector<uint8_t>> bufs(threads);
    std::atomic<bool> overflow{false};
    std::vector<std::vector<uint64_t>> local_off(threads);
    auto work = [&](uint32_t t) {
        uint32_t s0 = (uint32_t)((uint64_t)col->n_slots * t / threads);
        uint32_t s1 = (uint32_t)((uint64_t)col->n_slots * (t + 1) / threads);
        auto& buf = bufs[t];
        // room for the raw bytes of the thread's blocks and their headers, so
        // that the buffer does not move as it grows (compressed blocks are
        // smaller, literal-run blocks a few bytes larger)
        buf.reserve((size_t)(s1 - s0) * ((size_t)rows_per_block * 4 + rows_per_block / 64 + 256));
        std::vector<uint8_t> lz4_tmp;
        for (uint32_t s = s0; s < s1; ++s) {
            uint32_t c = s / col->blocks_per_chunk, j = s % col->blocks_per_chunk;
            uint64_t chunk_r0 = (uint64_t)c * rows_per_chunk;
            uint64_t chunk_r1 = std::min<uint64_t>(n_rows, chunk_r0 + rows_per_chunk);
            uint64_t r0 = chunk_r0 + (uint64_t)j * rows_per_block;
            if (r0 >= chunk_r1) continue;  // absent slot
            uint32_t rows = (uint32_t)std::min<uint64_t>(rows_per_block, chunk_r1 - r0);
            {
                int32_t mn = INT32_MAX, mx = INT32_MIN;
                for (uint32_t r = 0; r < rows; ++r) {
                    mn = std::min(mn, vals[r0 + r]);
                    mx = std::max(mx, vals[r0 + r]);
                }
                col->bmins[s] = mn;
                col->bmaxs[s] = mx;
            }
            size_t start = buf.size();
            size_t used = 0;
            if (codec == GX_CODEC_NONE) {
                buf.insert(buf.end(), (const uint8_t*)(vals + r0), (const uint8_t*)(vals + r0 + rows));
                used = (size_t)rows * 4;
            } else if (codec == GX_CODEC_LZ4) {
                uint32_t tmp_seg[2 * kMaxSegments];
                lz4_tmp.clear();
                used = min_match ? lz4_encode_block(vals + r0, rows, S, rows_per_block / S, min_match, depth, lz4_tmp,
                                                    tmp_seg, nullptr)
                                 : lz4_encode_block_auto(vals + r0, rows, S, rows_per_block / S, depth, lz4_tmp,
                                                         tmp_seg);
                if (used + 16 > kStageBytes) overflow = true;  // cannot happen for <= 16384 int32 rows
                if (S > 1) std::memcpy(&col->seg[(size_t)2 * S * s], tmp_seg, 8 * S);
                // place the block so that its first literal byte is 16-byte aligned
                // (buffers are concatenated at 16-byte multiples, so alignment here
                // is alignment in the payload)
                const long lit0 = lz4_first_literal(lz4_tmp.data(), lz4_tmp.size());
                if (lit0 >= 0) buf.resize(buf.size() + ((16 - (buf.size() + (size_t)lit0) % 16) % 16), 0);
                start = buf.size();
                buf.insert(buf.end(), lz4_tmp.begin(), lz4_tmp.end());
            } else {
                used = casc_encode_block(vals + r0, rows, rle, delta, bp, buf, &col->seg[(size_t)2 * S * s]);
            }
            buf.resize((buf.size() + kPayloadAlign - 1) & ~(size_t)(kPayloadAlign - 1), 0);
            col->blocks[s].offset = start;  // local, fixed up below
            col->blocks[s].comp_bytes = (uint32_t)used;
            col->blocks[s].n_rows = rows;
            local_off[t].push_back(s);
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < threads; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    if (overflow) return set_error(GX_ERR_INVALID, "an LZ4 block exceeds the %u-byte staging buffer", kStageBytes);
    // the per-thread buffers in thread order, each copied by its own thread
    std::vector<uint64_t> shift(threads + 1, 0);
    for (uint32_t t = 0; t < threads; ++t) shift[t + 1] = shift[t] + bufs[t].size();
    col->payload.assign(shift[threads] + kPayloadSlack, 0);
    auto place = [&](uint32_t t) {
        for (uint64_t s : local_off[t]) col->blocks[s].offset += shift[t];
        if (!bufs[t].empty()) std::memcpy(col->payload.data() + shift[t], bufs[t].data(), bufs[t].size());
        std::vector<uint8_t>().swap(bufs[t]);
    };
    pool.clear();
    for (uint32_t t = 1; t < threads; ++t) pool.emplace_back(place, t);
    place(0);
    for (auto& th : pool) th.join();
    col->n_blocks = 0;
    for (auto& b : col->blocks) col->n_blocks += b.n_rows ? 1 : 0;
    return GX_OK;
}

}  // namespace gx
