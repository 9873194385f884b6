// See system_build.hpp.
#include "system_build.hpp"

#include <omp.h>

#include <algorithm>
#include <cstdio>

#include "mh_darcy.h"
#include "mh_types.hpp"

namespace mh {

int local_edges(const MeshData &m, const Topology &t, int64_t e, int32_t *out) {
    int n = m.dim[e] + 1;
    int c = 0;
    for (int i = 0; i < n; ++i) out[c++] = t.side_edge[t.el_side_start[e] + i];
    for (int j = t.el_ngh_start[e]; j < t.el_ngh_start[e + 1]; ++j) out[c++] = t.ngh_edge[t.el_ngh[j]];
    return c;
}

void build_block_plan(HostSystem &hs, int target_blocks, HostSystem::Plan &plan) {
    const int n_inst = (int)hs.inst_row.size() - 1;
    const int64_t total = hs.n_tiles;
    plan = HostSystem::Plan();
    plan.inst_blk.assign(n_inst + 1, 0);
    for (int i = 0; i < n_inst; ++i) {
        const int64_t t0 = hs.inst_row[i] / hs.tile_rows, t1 = hs.inst_row[i + 1] / hs.tile_rows;
        const int64_t nt = t1 - t0;
        int64_t nb = (int64_t)((double)target_blocks * (double)nt / (double)total + 0.5);
        nb = std::max<int64_t>(1, std::min(nb, nt));
        plan.inst_blk[i] = (int32_t)plan.blk_inst.size();
        for (int64_t b = 0; b < nb; ++b) {
            plan.blk_inst.push_back(i);
            plan.blk_tile_begin.push_back((int32_t)(t0 + nt * b / nb));
            plan.blk_tile_end.push_back((int32_t)(t0 + nt * (b + 1) / nb));
        }
    }
    plan.inst_blk[n_inst] = (int32_t)plan.blk_inst.size();
}

void set_launch_shape(HostSystem &hs, int rows_per_thread, const int target_blocks[2]) {
    const int n_inst = (int)hs.inst_row.size() - 1;
    hs.rows_per_thread = rows_per_thread;
    hs.tile_rows = (int64_t)kTileRowsBase * rows_per_thread;
    hs.n_tiles = hs.n_rows / hs.tile_rows;
    hs.tile_inst.resize(hs.n_tiles);
    for (int i = 0; i < n_inst; ++i)
        for (int64_t tl = hs.inst_row[i] / hs.tile_rows; tl < hs.inst_row[i + 1] / hs.tile_rows; ++tl)
            hs.tile_inst[tl] = i;
    build_block_plan(hs, target_blocks[0], hs.plan[0]);
    build_block_plan(hs, target_blocks[1], hs.plan[1]);
}

int build_host_system(const MeshData &m, const Topology &t, const std::vector<int64_t> &inst_el,
                      int rows_per_thread, const int target_blocks[2], HostSystem &hs, std::string *err,
                      const ExtraBlocks *extra) {
    char msg[256];
    hs = HostSystem();
    hs.inst_el = inst_el;
    hs.rows_per_thread = rows_per_thread;
    hs.tile_rows = (int64_t)kTileRowsBase * rows_per_thread;
    const int64_t n_el = m.n_el, n_edges = t.n_edges();
    const int n_inst = (int)inst_el.size() - 1;

    // local block sizes and offsets
    hs.el_m.resize(n_el);
    hs.blk_off.resize(n_el);
    hs.rhs_off.resize(n_el);
    int64_t nb = 0, nr = 0;
    for (int64_t e = 0; e < n_el; ++e) {
        int d = m.dim[e];
        int k = t.el_ngh_start[e + 1] - t.el_ngh_start[e];
        int kmax = (d == 1) ? kMaxNgh1 : (d == 2 ? kMaxNgh2 : 0);
        if (k > kmax) {
            snprintf(msg, sizeof msg, "element %lld has %d VB neighbours (limit %d for dimension %d)",
                     (long long)e, k, kmax, d);
            if (err) *err = msg;
            return MH_ERR_TOPOLOGY;
        }
        int mm = d + 1 + k;
        hs.el_m[e] = mm;
        hs.blk_off[e] = nb;
        hs.rhs_off[e] = nr;
        nb += (int64_t)mm * mm;
        nr += mm;
        hs.dim_list[d].push_back((int32_t)e);
    }
    hs.n_blk = nb;
    hs.n_rhs_loc = nr;
    if (nb > INT32_MAX || nr > INT32_MAX) {
        if (err) *err = "mesh too large for 32-bit contribution indices";
        return MH_ERR_INVALID;
    }

    // instance edge ranges: edges are created while the instance's elements are visited,
    // so each instance owns a contiguous edge range
    hs.inst_edge.assign(n_inst + 1, 0);
    {
        std::vector<int32_t> owner(n_edges, -1);
        int32_t loc[16];
        for (int i = 0; i < n_inst; ++i)
            for (int64_t e = inst_el[i]; e < inst_el[i + 1]; ++e) {
                int c = local_edges(m, t, e, loc);
                for (int l = 0; l < c; ++l) {
                    if (owner[loc[l]] >= 0 && owner[loc[l]] != i) {
                        if (err) *err = "instances share an edge";
                        return MH_ERR_INVALID;
                    }
                    owner[loc[l]] = i;
                }
            }
        for (int64_t g = 0; g < n_edges; ++g) {
            if (owner[g] < 0) {
                if (err) *err = "edge without an element";
                return MH_ERR_TOPOLOGY;
            }
            if (g > 0 && owner[g] < owner[g - 1]) {
                if (err) *err = "instance edge ranges are not contiguous";
                return MH_ERR_INVALID;
            }
        }
        int64_t g = 0;
        for (int i = 0; i < n_inst; ++i) {
            hs.inst_edge[i] = g;
            while (g < n_edges && owner[g] == i) ++g;
        }
        hs.inst_edge[n_inst] = g;
    }

    // padded solver rows per instance: a multiple of kPadRows, so tiles of 256*R rows never
    // straddle instances for any R in {1, 2, 4} and R can be retuned without a rebuild
    hs.inst_row.assign(n_inst + 1, 0);
    for (int i = 0; i < n_inst; ++i) {
        int64_t ne = hs.inst_edge[i + 1] - hs.inst_edge[i];
        int64_t pad = ((ne + kPadRows - 1) / kPadRows) * kPadRows;
        if (pad == 0) pad = kPadRows;
        hs.inst_row[i + 1] = hs.inst_row[i] + pad;
    }
    hs.n_rows = hs.inst_row[n_inst];
    hs.n_slices = hs.n_rows / kSliceRowsHost;
    hs.edge_row.resize(n_edges);
    hs.row_edge.assign(hs.n_rows, -1);
    for (int i = 0; i < n_inst; ++i)
        for (int64_t g = hs.inst_edge[i]; g < hs.inst_edge[i + 1]; ++g) {
            int64_t r = hs.inst_row[i] + (g - hs.inst_edge[i]);
            hs.edge_row[g] = (int32_t)r;
            hs.row_edge[r] = (int32_t)g;
        }
    set_launch_shape(hs, rows_per_thread, target_blocks);

    // symmetric pattern: every pair of an element's local edges
    // (each row is sorted and deduplicated below, so the rows are filled in parallel in any order)
    std::vector<int64_t> cnt(hs.n_rows + 1, 0);
    int32_t loc[16];
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n_el; ++e) {
        int32_t lc[16];
        int c = local_edges(m, t, e, lc);
        for (int a = 0; a < c; ++a) {
#pragma omp atomic
            cnt[hs.edge_row[lc[a]] + 1] += c;
        }
    }
    for (int64_t r = 0; r < hs.n_rows; ++r)
        if (hs.row_edge[r] < 0) cnt[r + 1] += 1;
    if (extra)
        for (const auto &g : extra->edges)
            for (int32_t a : g) cnt[hs.edge_row[a] + 1] += (int64_t)g.size();
    for (int64_t r = 0; r < hs.n_rows; ++r) cnt[r + 1] += cnt[r];
    std::vector<int32_t> raw(cnt[hs.n_rows]);
    {
        std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
#pragma omp parallel for schedule(static)
        for (int64_t e = 0; e < n_el; ++e) {
            int32_t lc[16];
            int c = local_edges(m, t, e, lc);
            for (int a = 0; a < c; ++a) {
                const int64_t ra = hs.edge_row[lc[a]];
                int64_t pos;
#pragma omp atomic capture
                {
                    pos = fill[ra];
                    fill[ra] += c;
                }
                for (int b = 0; b < c; ++b) raw[pos + b] = hs.edge_row[lc[b]];
            }
        }
        for (int64_t r = 0; r < hs.n_rows; ++r)
            if (hs.row_edge[r] < 0) raw[fill[r]++] = (int32_t)r;
        if (extra)
            for (const auto &g : extra->edges)
                for (int32_t a : g) {
                    const int64_t ra = hs.edge_row[a];
                    for (int32_t b : g) raw[fill[ra]++] = hs.edge_row[b];
                }
    }
    hs.row_ptr.assign(hs.n_rows + 1, 0);
    std::vector<int64_t> len(hs.n_rows);
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t r = 0; r < hs.n_rows; ++r) {
        auto b = raw.begin() + cnt[r], e = raw.begin() + cnt[r + 1];
        std::sort(b, e);
        len[r] = std::unique(b, e) - b;
    }
    for (int64_t r = 0; r < hs.n_rows; ++r) hs.row_ptr[r + 1] = hs.row_ptr[r] + len[r];
    hs.row_col.resize(hs.row_ptr[hs.n_rows]);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < hs.n_rows; ++r)
        std::copy(raw.begin() + cnt[r], raw.begin() + cnt[r] + len[r], hs.row_col.begin() + hs.row_ptr[r]);
    hs.nnz = 0;
    for (int64_t r = 0; r < hs.n_rows; ++r)
        if (hs.row_edge[r] >= 0) hs.nnz += len[r];
    raw.clear();
    raw.shrink_to_fit();

    // SELL-C-sigma with C = 32 (sigma = 1: the mesh ordering already keeps row lengths even)
    hs.slice_off.assign(hs.n_slices + 1, 0);
    for (int64_t s = 0; s < hs.n_slices; ++s) {
        int64_t w = 0;
        for (int l = 0; l < kSliceRowsHost; ++l) w = std::max(w, len[s * kSliceRowsHost + l]);
        hs.slice_off[s + 1] = hs.slice_off[s] + w * kSliceRowsHost;
    }
    hs.n_slots = hs.slice_off[hs.n_slices];
    if (hs.n_slots > INT32_MAX) {
        if (err) *err = "system too large for 32-bit slot indices";
        return MH_ERR_INVALID;
    }
    hs.sell_col.resize(hs.n_slots);
    hs.diag_slot.resize(hs.n_rows);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < hs.n_rows; ++r) {
        int64_t s = r / kSliceRowsHost, lane = r % kSliceRowsHost;
        int64_t off = hs.slice_off[s], w = (hs.slice_off[s + 1] - off) / kSliceRowsHost;
        for (int64_t j = 0; j < w; ++j) {
            int32_t c = (j < len[r]) ? hs.row_col[hs.row_ptr[r] + j] : (int32_t)r;
            hs.sell_col[off + j * kSliceRowsHost + lane] = c;
            if (j < len[r] && c == r) hs.diag_slot[r] = (int32_t)(off + j * kSliceRowsHost + lane);
        }
    }
    auto slot_of = [&](int64_t r, int32_t c) -> int64_t {
        auto b = hs.row_col.begin() + hs.row_ptr[r], e = hs.row_col.begin() + hs.row_ptr[r + 1];
        int64_t j = std::lower_bound(b, e, c) - b;
        return hs.slice_off[r / kSliceRowsHost] + j * kSliceRowsHost + r % kSliceRowsHost;
    };

    // the extra blocks' values summed per slot in group order (the host does it once)
    if (extra) {
        std::vector<std::pair<int32_t, double>> sv;
        for (size_t k = 0; k < extra->edges.size(); ++k) {
            const auto &g = extra->edges[k];
            const size_t q = g.size();
            for (size_t a = 0; a < q; ++a)
                for (size_t b = 0; b < q; ++b)
                    sv.push_back({(int32_t)slot_of(hs.edge_row[g[a]], hs.edge_row[g[b]]), extra->vals[k][a * q + b]});
        }
        std::stable_sort(sv.begin(), sv.end(), [](const auto &x, const auto &y) { return x.first < y.first; });
        for (const auto &e : sv) {
            if (hs.add_slot.empty() || hs.add_slot.back() != e.first) {
                hs.add_slot.push_back(e.first);
                hs.add_val.push_back(0.0);
            }
            hs.add_val.back() += e.second;
        }
    }

    // contributions: element blocks -> slots, element rhs -> rows, in element order (the
    // device sums each slot's contributions in list order).  The slot of every block entry
    // (a binary search in its row) is found in parallel for a chunk of elements; counting and
    // filling then walk the chunk in element order.
    constexpr int64_t kChunk = 1 << 18;
    std::vector<int64_t> coff(kChunk + 1);
    std::vector<int32_t> cslot;  // n_slots < 2^31 (checked above)
    auto chunk_slots = [&](int64_t e0, int64_t e1) {
        coff[0] = 0;
        for (int64_t e = e0; e < e1; ++e) {
            const int64_t c = m.dim[e] + 1 + (t.el_ngh_start[e + 1] - t.el_ngh_start[e]);  // local_edges' count
            coff[e - e0 + 1] = coff[e - e0] + c * c;
        }
        cslot.resize(coff[e1 - e0]);
#pragma omp parallel for schedule(static)
        for (int64_t e = e0; e < e1; ++e) {
            int32_t lc[16];
            const int c = local_edges(m, t, e, lc);
            int64_t o = coff[e - e0];
            for (int a = 0; a < c; ++a) {
                const int64_t ra = hs.edge_row[lc[a]];
                for (int b = 0; b < c; ++b) cslot[o++] = (int32_t)slot_of(ra, hs.edge_row[lc[b]]);
            }
        }
    };
    hs.slot_cstart.assign(hs.n_slots + 1, 0);
    hs.row_cstart.assign(hs.n_rows + 1, 0);
    for (int64_t e0 = 0; e0 < n_el; e0 += kChunk) {
        const int64_t e1 = std::min(n_el, e0 + kChunk);
        chunk_slots(e0, e1);
        for (int64_t e = e0; e < e1; ++e) {
            int c = local_edges(m, t, e, loc);
            const int64_t o = coff[e - e0];
            for (int a = 0; a < c; ++a) {
                hs.row_cstart[hs.edge_row[loc[a]] + 1]++;
                for (int b = 0; b < c; ++b) hs.slot_cstart[cslot[o + (int64_t)a * c + b] + 1]++;
            }
        }
    }
    for (int64_t s = 0; s < hs.n_slots; ++s) hs.slot_cstart[s + 1] += hs.slot_cstart[s];
    for (int64_t r = 0; r < hs.n_rows; ++r) hs.row_cstart[r + 1] += hs.row_cstart[r];
    hs.slot_cidx.resize(hs.slot_cstart[hs.n_slots]);
    hs.row_cidx.resize(hs.row_cstart[hs.n_rows]);
    {
        // every thread owns a contiguous range of slots and of rows and walks the chunk in element
        // order, writing only its own lists: each list keeps the element order
        std::vector<int32_t> sf(hs.slot_cstart.begin(), hs.slot_cstart.end() - 1);
        std::vector<int32_t> rf(hs.row_cstart.begin(), hs.row_cstart.end() - 1);
        for (int64_t e0 = 0; e0 < n_el; e0 += kChunk) {
            const int64_t e1 = std::min(n_el, e0 + kChunk);
            chunk_slots(e0, e1);
#pragma omp parallel
            {
                const int nt = omp_get_num_threads(), th = omp_get_thread_num();
                const int64_t s_lo = hs.n_slots * th / nt, s_hi = hs.n_slots * (th + 1) / nt;
                const int64_t r_lo = hs.n_rows * th / nt, r_hi = hs.n_rows * (th + 1) / nt;
                int32_t lc[16];
                for (int64_t e = e0; e < e1; ++e) {
                    const int c = local_edges(m, t, e, lc);
                    const int64_t o = coff[e - e0];
                    for (int a = 0; a < c; ++a) {
                        const int64_t ra = hs.edge_row[lc[a]];
                        if (ra >= r_lo && ra < r_hi) hs.row_cidx[rf[ra]++] = (int32_t)(hs.rhs_off[e] + a);
                        for (int b = 0; b < c; ++b) {
                            const int64_t sl = cslot[o + (int64_t)a * c + b];
                            if (sl >= s_lo && sl < s_hi)
                                hs.slot_cidx[sf[sl]++] = (int32_t)(hs.blk_off[e] + (int64_t)a * c + b);
                        }
                    }
                }
            }
        }
    }
    return MH_OK;
}

int build_host_system_csr(int64_t n, const int32_t *row_ptr, const int32_t *col, int rows_per_thread,
                          const int target_blocks[2], HostSystem &hs, std::string *err) {
    hs = HostSystem();
    if (n <= 0 || !row_ptr || !col || row_ptr[0] != 0) {
        if (err) *err = "empty system or invalid row pointers";
        return MH_ERR_INVALID;
    }
    for (int64_t r = 0; r < n; ++r) {
        bool diag = false;
        if (row_ptr[r + 1] < row_ptr[r]) {
            if (err) *err = "row pointers decrease";
            return MH_ERR_INVALID;
        }
        for (int32_t k = row_ptr[r]; k < row_ptr[r + 1]; ++k) {
            if (col[k] < 0 || col[k] >= n || (k > row_ptr[r] && col[k] <= col[k - 1])) {
                char msg[160];
                snprintf(msg, sizeof msg, "row %lld: columns out of range, unsorted or repeated", (long long)r);
                if (err) *err = msg;
                return MH_ERR_INVALID;
            }
            diag |= col[k] == r;
        }
        if (!diag) {
            char msg[160];
            snprintf(msg, sizeof msg, "row %lld has no diagonal entry", (long long)r);
            if (err) *err = msg;
            return MH_ERR_INVALID;
        }
    }
    hs.inst_el = {0, 0};
    hs.inst_edge = {0, n};
    const int64_t pad = ((n + kPadRows - 1) / kPadRows) * kPadRows;
    hs.inst_row = {0, pad};
    hs.n_rows = pad;
    hs.n_slices = pad / kSliceRowsHost;
    hs.edge_row.resize(n);
    hs.row_edge.assign(pad, -1);
    for (int64_t g = 0; g < n; ++g) {
        hs.edge_row[g] = (int32_t)g;
        hs.row_edge[g] = (int32_t)g;
    }
    set_launch_shape(hs, rows_per_thread, target_blocks);
    hs.row_ptr.assign(pad + 1, 0);
    for (int64_t r = 0; r < pad; ++r) hs.row_ptr[r + 1] = hs.row_ptr[r] + (r < n ? row_ptr[r + 1] - row_ptr[r] : 1);
    hs.row_col.resize(hs.row_ptr[pad]);
    for (int64_t r = 0; r < pad; ++r) {
        if (r < n)
            std::copy(col + row_ptr[r], col + row_ptr[r + 1], hs.row_col.begin() + hs.row_ptr[r]);
        else
            hs.row_col[hs.row_ptr[r]] = (int32_t)r;  // padding rows: a unit diagonal
    }
    hs.nnz = row_ptr[n];
    hs.slice_off.assign(hs.n_slices + 1, 0);
    for (int64_t sl = 0; sl < hs.n_slices; ++sl) {
        int64_t w = 0;
        for (int l = 0; l < kSliceRowsHost; ++l) {
            const int64_t r = sl * kSliceRowsHost + l;
            w = std::max(w, hs.row_ptr[r + 1] - hs.row_ptr[r]);
        }
        hs.slice_off[sl + 1] = hs.slice_off[sl] + w * kSliceRowsHost;
    }
    hs.n_slots = hs.slice_off[hs.n_slices];
    if (hs.n_slots > INT32_MAX) {
        if (err) *err = "system too large for 32-bit slot indices";
        return MH_ERR_INVALID;
    }
    hs.sell_col.resize(hs.n_slots);
    hs.diag_slot.resize(pad);
    hs.csr_slot.resize(hs.nnz);
    for (int64_t r = 0; r < pad; ++r) {
        const int64_t sl = r / kSliceRowsHost, lane = r % kSliceRowsHost;
        const int64_t off = hs.slice_off[sl], w = (hs.slice_off[sl + 1] - off) / kSliceRowsHost;
        const int64_t len = hs.row_ptr[r + 1] - hs.row_ptr[r];
        for (int64_t j = 0; j < w; ++j) {
            const int64_t slot = off + j * kSliceRowsHost + lane;
            const int32_t c = j < len ? hs.row_col[hs.row_ptr[r] + j] : (int32_t)r;
            hs.sell_col[slot] = c;
            if (j < len && c == r) hs.diag_slot[r] = (int32_t)slot;
            if (j < len && r < n) hs.csr_slot[hs.row_ptr[r] + j] = (int32_t)slot;
        }
    }
    hs.slot_cstart.assign(hs.n_slots + 1, 0);
    hs.row_cstart.assign(pad + 1, 0);
    return MH_OK;
}

}  // namespace mh
