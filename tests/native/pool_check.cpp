// Drives gsc_b200::RangePool from stdin for the pool test:
//   c <capacity>        reset
//   a <bytes>           alloc; prints the offset or -1
//   f <offset> <bytes>  release
//   s                   prints used, largest free range, free range count
#include <cstdint>
#include <iostream>
#include <string>

#include "gsc_pool.hpp"

int main() {
    gsc_b200::RangePool pool;
    std::string op;
    while (std::cin >> op) {
        if (op == "c") {
            uint64_t cap;
            std::cin >> cap;
            pool.reset(cap);
        } else if (op == "a") {
            uint64_t n;
            std::cin >> n;
            const uint64_t off = pool.alloc(n);
            if (off == gsc_b200::RangePool::kNone)
                std::cout << -1 << "\n";
            else
                std::cout << off << "\n";
        } else if (op == "f") {
            uint64_t off, n;
            std::cin >> off >> n;
            pool.release(off, n);
        } else if (op == "s") {
            std::cout << pool.used() << " " << pool.largest_free() << " " << pool.free_ranges() << "\n";
        }
    }
    return 0;
}
