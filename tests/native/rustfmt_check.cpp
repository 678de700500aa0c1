// Reads doubles (hex bit patterns, one per line) from stdin and prints, per
// value, the driver's Rust formats separated by '|': {:.4} {:.6} {:.3e}
// {:.8e} {:e} {}.  Test infrastructure for tests/test_driver_cpu.py.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <string>

#include "rustfmt.h"

int main() {
    std::string line;
    while (std::getline(std::cin, line)) {
        if (line.empty()) continue;
        const uint64_t bits = std::stoull(line, nullptr, 16);
        double x;
        std::memcpy(&x, &bits, 8);
        std::cout << rf::fixed(x, 4) << '|' << rf::fixed(x, 6) << '|' << rf::exp(x, 3) << '|' << rf::exp(x, 8)
                  << '|' << rf::exp_short(x) << '|' << rf::display(x) << '\n';
    }
    return 0;
}
