// Randomised check of nsat::LruMap (naivesat_b200/csrc/lru.h) against a
// plain model: a vector of (key, value) pairs, most recently used first.
// Built and run by tests/test_abi_cpu.py; exits 0 when every step agrees.
#include <cstdio>
#include <cstdint>
#include <vector>

#include "lru.h"

namespace {

struct Model {
    size_t cap;
    std::vector<std::pair<int, int>> items;   // most recently used first

    int* find(int k) {
        for (size_t i = 0; i < items.size(); i++)
            if (items[i].first == k) {
                auto e = items[i];
                items.erase(items.begin() + (long)i);
                items.insert(items.begin(), e);
                return &items[0].second;
            }
        return nullptr;
    }
    void put(int k, int v, std::vector<int>* evicted) {
        for (size_t i = 0; i < items.size(); i++)
            if (items[i].first == k) {
                evicted->push_back(items[i].second);
                items.erase(items.begin() + (long)i);
                items.insert(items.begin(), {k, v});
                return;
            }
        items.insert(items.begin(), {k, v});
        trim(evicted);
    }
    void trim(std::vector<int>* evicted) {
        while (items.size() > cap) {
            evicted->push_back(items.back().second);
            items.pop_back();
        }
    }
};

uint64_t rng_state = 0x9E3779B97F4A7C15ull;
uint32_t next_u32() {
    rng_state ^= rng_state << 13;
    rng_state ^= rng_state >> 7;
    rng_state ^= rng_state << 17;
    return (uint32_t)rng_state;
}

}  // namespace

int main() {
    for (size_t cap : {1u, 2u, 3u, 7u, 32u}) {
        nsat::LruMap<int, int> lru(cap);
        Model m{cap, {}};
        int value = 0;
        for (int step = 0; step < 20000; step++) {
            const int k = (int)(next_u32() % (3 * cap + 2));
            const uint32_t op = next_u32() % 10;
            if (op < 5) {
                int* a = lru.find(k);
                int* b = m.find(k);
                if ((a == nullptr) != (b == nullptr) || (a && *a != *b)) {
                    printf("cap %zu step %d: find(%d) differs\n", cap, step, k);
                    return 1;
                }
            } else if (op < 9) {
                std::vector<int> ea, eb;
                lru.put(k, ++value, &ea);
                m.put(k, value, &eb);
                if (ea != eb) {
                    printf("cap %zu step %d: put(%d) evicted differently\n", cap, step, k);
                    return 1;
                }
            } else {
                const size_t c2 = 1 + next_u32() % (2 * cap);
                std::vector<int> ea, eb;
                lru.set_capacity(c2, &ea);
                m.cap = c2;
                m.trim(&eb);
                if (ea != eb) {
                    printf("cap %zu step %d: set_capacity(%zu) evicted differently\n", cap, step, c2);
                    return 1;
                }
            }
            if (lru.size() != m.items.size() || lru.size() > lru.capacity()) {
                printf("cap %zu step %d: size %zu vs %zu\n", cap, step, lru.size(), m.items.size());
                return 1;
            }
        }
    }
    printf("ok\n");
    return 0;
}
