// CPU check of the launch-size arithmetic (gkm-dns_b200/csrc/gks_limits.h):
// for several SM counts and field sizes, every helper grid stays within its
// per-SM cap, the statistics grid never has more blocks than the partial-sum
// buffer sized from the same SM count holds, and the per-context address
// cache re-resolves exactly when the context id changes.  Prints "ok" and
// exits 0, or names the first violated limit and exits 1.
#include "gks_limits.h"

#include <cstdio>
#include <initializer_list>

static int fails = 0;
#define EXPECT(c)                                                      \
    do {                                                               \
        if (!(c)) {                                                    \
            std::printf("FAIL line %d: %s\n", __LINE__, #c);           \
            ++fails;                                                   \
        }                                                              \
    } while (0)

int main()
{
    const int nsms[] = {1, 2, 7, 66, 108, 132, 148, 160, 264};
    const long long ncs[] = {4, 8, 24, 64, 96, 128, 256, 512, 1024};
    for (int nsm : nsms)
        for (long long nc : ncs) {
            const long long ncell = nc * nc * nc, nt = nc + 6;
            for (long long items : {ncell, nt * nt * nt}) {
                const int g = gks::helper_grid(items, 256, nsm);
                EXPECT(g >= 1);
                EXPECT(g <= nsm * gks::kHelperBlocksPerSm);
                EXPECT((long long)g * 256 >= items || g == nsm * gks::kHelperBlocksPerSm);
            }
            const int sg = gks::stats_grid(ncell, 256, nsm);
            EXPECT(sg >= 1);
            EXPECT(sg <= nsm * gks::kStatsBlocksPerSm);
            EXPECT((size_t)sg * gks::kStatsSums <= gks::stats_partial_elems(nsm));
        }
    // the address cache: resolve once per (device, context), again after the context changes
    gks::ContextAddressCache<4> cache;
    int calls = 0;
    char a0, a1;
    void *next = &a0;
    auto resolve = [&](void **p) {
        ++calls;
        *p = next;
        return 0;
    };
    void *got = nullptr;
    EXPECT(cache.get(0, 11, resolve, &got) == 0 && got == &a0 && calls == 1);
    EXPECT(cache.get(0, 11, resolve, &got) == 0 && got == &a0 && calls == 1);
    next = &a1;
    EXPECT(cache.get(0, 12, resolve, &got) == 0 && got == &a1 && calls == 2); // new context: looked up again
    EXPECT(cache.get(1, 12, resolve, &got) == 0 && got == &a1 && calls == 3); // another device
    EXPECT(cache.get(0, 12, resolve, &got) == 0 && got == &a1 && calls == 3);
    EXPECT(cache.get(4, 12, resolve, &got) != 0);                              // device out of range
    EXPECT(cache.get(-1, 12, resolve, &got) != 0);
    auto broken = [&](void **p) {
        *p = nullptr;
        return 7;
    };
    EXPECT(cache.get(2, 12, broken, &got) == 7);
    EXPECT(cache.get(2, 12, resolve, &got) == 0 && got == &a1); // a failed lookup is not cached
    if (fails) return 1;
    std::printf("ok\n");
    return 0;
}
