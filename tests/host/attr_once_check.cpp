// Host check of cps::attr_once_per_device (cpsfdtd_b200/csrc/attr_once.h)
// with a fake device switch and a fake attribute call: the attribute is set
// once per device, again on each device a thread moves to, retried after a
// failure, set on every call for device ordinals past 64, and under many
// threads racing on 8 devices every device ends up set.  Exits 0 and prints
// "ok" when every case holds.
#include <stdio.h>
#include <stdlib.h>

#include <atomic>
#include <thread>
#include <vector>

#include "attr_once.h"

static thread_local int t_dev = 0;
static std::atomic<int> calls[128];
static std::atomic<int> fail_next{0};

static int get_dev(int *d)
{
    *d = t_dev;
    return 0;
}

static int apply()
{
    calls[t_dev].fetch_add(1);
    if (fail_next.load() > 0) {
        fail_next.fetch_sub(1);
        return 1;  // a failing attribute call
    }
    return 0;
}

#define CHECK(c)                                                    \
    do {                                                            \
        if (!(c)) {                                                 \
            printf("FAILED line %d: %s\n", __LINE__, #c);           \
            return 1;                                               \
        }                                                           \
    } while (0)

int main()
{
    std::atomic<uint64_t> done{0};
    // once on device 0
    t_dev = 0;
    CHECK(cps::attr_once_per_device(done, get_dev, apply) == 0);
    CHECK(cps::attr_once_per_device(done, get_dev, apply) == 0);
    CHECK(calls[0] == 1);
    // a second device needs its own call
    t_dev = 3;
    CHECK(cps::attr_once_per_device(done, get_dev, apply) == 0);
    CHECK(calls[3] == 1);
    CHECK(done.load() == ((1ull << 0) | (1ull << 3)));
    // a failure is returned, leaves the device unset, and is retried
    t_dev = 5;
    fail_next = 1;
    CHECK(cps::attr_once_per_device(done, get_dev, apply) == 1);
    CHECK((done.load() & (1ull << 5)) == 0);
    CHECK(cps::attr_once_per_device(done, get_dev, apply) == 0);
    CHECK(calls[5] == 2);
    CHECK(cps::attr_once_per_device(done, get_dev, apply) == 0);
    CHECK(calls[5] == 2);
    // ordinals past the mask are set on every call
    t_dev = 70;
    CHECK(cps::attr_once_per_device(done, get_dev, apply) == 0);
    CHECK(cps::attr_once_per_device(done, get_dev, apply) == 0);
    CHECK(calls[70] == 2);
    // a failing device query is passed through without an attribute call
    auto bad_dev = [](int *) { return 7; };
    CHECK(cps::attr_once_per_device(done, bad_dev, apply) == 7);
    // many threads on 8 devices: every device set, each at least once
    std::atomic<uint64_t> done2{0};
    for (auto &c : calls) c = 0;
    std::vector<std::thread> th;
    for (int t = 0; t < 32; ++t)
        th.emplace_back([&, t] {
            for (int r = 0; r < 1000; ++r) {
                t_dev = (t + r) % 8;
                if (cps::attr_once_per_device(done2, get_dev, apply) != 0) abort();
            }
        });
    for (auto &x : th) x.join();
    CHECK(done2.load() == 0xffull);
    for (int d = 0; d < 8; ++d) CHECK(calls[d] >= 1 && calls[d] <= 32);
    printf("ok\n");
    return 0;
}
