// Host check of cps::tfsf_assemble (cpsfdtd_b200/csrc/tfsf_csr.h) against a
// serial restatement of the same ordering: counting sort of all items by
// plane (strips in order, items in order), stable sort by key within each
// plane, one target per run of equal keys.  Exits 0 and prints "ok" when every
// case gives byte-identical target and contribution arrays.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <random>
#include <thread>
#include <vector>

#include "tfsf_csr.h"

struct Contrib {
    double delay, profile, coef;
    int32_t face, pad;
};
struct Target {
    int64_t idx;
    int32_t comp, start, count, face;
};
struct Item {
    int64_t key;
    Contrib c;
};

static void pfor(int n, auto f)
{
    const int parts = std::min(8, n);
    if (parts <= 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 1; t < parts; ++t)
        th.emplace_back([&f, n, t, parts] { f((int)((int64_t)n * t / parts), (int)((int64_t)n * (t + 1) / parts)); });
    f(0, n / parts);
    for (std::thread &x : th) x.join();
}

static void serial(const std::vector<std::vector<Item>> &strips, int nz1, int64_t pxy, std::vector<Target> &tg,
                   std::vector<Contrib> &ct)
{
    std::vector<Item> items;
    for (int k = 0; k < nz1; ++k) {
        const size_t first = items.size();
        for (const auto &st : strips)
            for (const Item &it : st)
                if (it.key / 8 / pxy == k) items.push_back(it);
        std::stable_sort(items.begin() + first, items.end(), [](const Item &a, const Item &b) { return a.key < b.key; });
    }
    for (size_t q = 0; q < items.size();) {
        size_t r = q;
        while (r < items.size() && items[r].key == items[q].key) ct.push_back(items[r++].c);
        Target t;
        memset(&t, 0, sizeof(t));
        t.idx = items[q].key / 8;
        t.comp = (int32_t)(items[q].key % 8);
        t.start = (int32_t)q;
        t.count = (int32_t)(r - q);
        t.face = items[q].c.face;
        tg.push_back(t);
        q = r;
    }
}

static bool one_case(const char *name, std::vector<std::vector<Item>> strips, int nz1, int64_t pxy)
{
    std::vector<Target> ta, tb;
    std::vector<Contrib> ca, cb;
    serial(strips, nz1, pxy, ta, ca);
    cps::tfsf_assemble(strips, nz1, pxy, [](int n, auto f) { pfor(n, f); }, tb, cb);
    const bool ok = ta.size() == tb.size() && ca.size() == cb.size() &&
                    (ta.empty() || memcmp(ta.data(), tb.data(), ta.size() * sizeof(Target)) == 0) &&
                    (ca.empty() || memcmp(ca.data(), cb.data(), ca.size() * sizeof(Contrib)) == 0);
    printf("%-28s %7zu targets %7zu contributions: %s\n", name, tb.size(), cb.size(), ok ? "same" : "DIFFERENT");
    return ok;
}

static Item item(int64_t cell, int comp, int face, int seq)
{
    Item it;
    memset(&it, 0, sizeof(it));
    it.key = cell * 8 + comp;
    it.c.delay = seq;
    it.c.profile = 0.5 * seq;
    it.c.coef = face;
    it.c.face = face;
    return it;
}

int main()
{
    bool ok = true;
    const int nz1 = 33;
    const int64_t pxy = 64 * 33;
    std::mt19937_64 rng(20261204);
    // random strips with many keys shared between strips (box edges and corners)
    for (int trial = 0; trial < 8; ++trial) {
        std::vector<std::vector<Item>> strips(12);
        int seq = 0;
        for (int s = 0; s < 12; ++s) {
            const int n = (int)(rng() % 2500);
            for (int q = 0; q < n; ++q)
                strips[s].push_back(item((int64_t)(rng() % nz1) * pxy + (int64_t)(rng() % 150), (int)(rng() % 6), s, seq++));
        }
        char name[64];
        snprintf(name, sizeof(name), "random strips %d", trial);
        ok &= one_case(name, strips, nz1, pxy);
    }
    // empty input, and strips that are all empty but one
    ok &= one_case("no strips", std::vector<std::vector<Item>>(), nz1, pxy);
    {
        std::vector<std::vector<Item>> strips(12);
        strips[7].push_back(item(5 * pxy + 3, 2, 7, 0));
        ok &= one_case("one item", strips, nz1, pxy);
    }
    // every item in one plane and one cell: a single target with every strip's
    // contributions in strip order
    {
        std::vector<std::vector<Item>> strips(12);
        for (int s = 0; s < 12; ++s)
            for (int q = 0; q < 3; ++q) strips[s].push_back(item(9 * pxy + 40, 1, s, s * 3 + q));
        ok &= one_case("one cell, every strip", strips, nz1, pxy);
    }
    // the last plane only, keys descending within each strip
    {
        std::vector<std::vector<Item>> strips(12);
        int seq = 0;
        for (int s = 0; s < 12; ++s)
            for (int q = 200; q > 0; --q) strips[s].push_back(item((nz1 - 1) * pxy + q, s % 6, s, seq++));
        ok &= one_case("last plane, descending keys", strips, nz1, pxy);
    }
    puts(ok ? "ok" : "FAILED");
    return ok ? 0 : 1;
}
