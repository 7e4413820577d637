// tfsf_csr.h -- assembly of the TF/SF injection tables (host code, no CUDA).
//
// The TF/SF set-up (TF_SF.cpp:29-959 restated in cps_tfsf_init) produces one
// contribution per (face, point, component) in twelve strips, each strip
// being one (face, correction) pair in the reference's face order.  The
// device applies them per target (cell, component) in CSR form: targets
// sorted by device index, each owning the run of its contributions in the
// reference's face order (a cell on a box edge or corner receives several).
//
// Item:    { int64_t key;  // cell index * 8 + component
//            Contrib c; }  // c.face is the face of the contribution
// Target:  { int64_t idx; int32_t comp, start, count, face; }
//
// The result equals a serial counting sort of all items by plane (strips in
// order, each strip's items in order), a stable sort by key within each
// plane, and one target per run of equal keys whose contributions start at
// the run's first item.  Every step here runs per strip or per plane through
// `parallel_for(n, f)`, which calls f(begin, end) on disjoint ranges of [0, n).
#pragma once

#include <stddef.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

namespace cps {

template <typename Item, typename Target, typename Contrib, typename ParallelFor>
void tfsf_assemble(std::vector<std::vector<Item>> &strips, int nz1, int64_t pxy, ParallelFor &&parallel_for,
                   std::vector<Target> &tg, std::vector<Contrib> &ct)
{
    const int ns = (int)strips.size();
    auto plane_of = [pxy](const Item &it) { return (size_t)(it.key / 8 / pxy); };
    std::vector<std::vector<size_t>> off(ns, std::vector<size_t>(nz1, 0));  // counts, then first slots
    parallel_for(ns, [&](int s0, int s1) {
        for (int st = s0; st < s1; ++st)
            for (const Item &it : strips[st]) off[st][plane_of(it)]++;
    });
    std::vector<size_t> start(nz1 + 1, 0);
    for (int k = 0; k < nz1; ++k) {
        size_t at = start[k];
        for (int st = 0; st < ns; ++st) {
            const size_t c = off[st][k];
            off[st][k] = at;
            at += c;
        }
        start[k + 1] = at;
    }
    std::vector<Item> items(start[nz1]);
    parallel_for(ns, [&](int s0, int s1) {
        for (int st = s0; st < s1; ++st) {
            std::vector<size_t> &o = off[st];
            for (const Item &it : strips[st]) items[o[plane_of(it)]++] = it;
        }
    });
    strips.clear();
    parallel_for(nz1, [&](int k0, int k1) {
        for (int k = k0; k < k1; ++k)
            std::stable_sort(items.begin() + start[k], items.begin() + start[k + 1],
                             [](const Item &a, const Item &b) { return a.key < b.key; });
    });
    // one target per run of equal keys (a run never crosses a plane)
    std::vector<size_t> tg_at(nz1 + 1, 0);
    parallel_for(nz1, [&](int k0, int k1) {
        for (int k = k0; k < k1; ++k) {
            size_t n = 0;
            for (size_t q = start[k]; q < start[k + 1]; ++q) n += q == start[k] || items[q].key != items[q - 1].key;
            tg_at[k + 1] = n;
        }
    });
    for (int k = 0; k < nz1; ++k) tg_at[k + 1] += tg_at[k];
    tg.assign(tg_at[nz1], Target{});
    ct.assign(items.size(), Contrib{});
    parallel_for(nz1, [&](int k0, int k1) {
        for (int k = k0; k < k1; ++k) {
            size_t t = tg_at[k];
            for (size_t q = start[k]; q < start[k + 1];) {
                size_t r = q;
                while (r < start[k + 1] && items[r].key == items[q].key) {
                    ct[r] = items[r].c;
                    ++r;
                }
                Target &tt = tg[t++];
                tt.idx = items[q].key / 8;
                tt.comp = (int)(items[q].key % 8);
                tt.start = (int32_t)q;
                tt.count = (int32_t)(r - q);
                tt.face = items[q].c.face;
                q = r;
            }
        }
    });
}

}  // namespace cps
