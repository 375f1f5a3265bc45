// Host build of zdx_pyset.cuh for tests/test_pyset_cpu.py.  Reads commands from stdin and prints one
// line per command:
//   S n k_1 .. k_n        the set order of the distinct ints k added in order
#include <cstdio>
#include <vector>

#include "zdx_pyset.cuh"

int main() {
    char cmd;
    int n;
    while (std::scanf(" %c %d", &cmd, &n) == 2) {
        if (cmd == 'S') {
            std::vector<int> keys(n), tab(8 * (size_t)n + 8), old((size_t)n + 1);
            for (int q = 0; q < n; ++q) std::scanf("%d", &keys[q]);
            bool ok = true;
            const unsigned mask = zdx::pyset_build(keys.data(), n, tab.data(), old.data(), &ok);
            std::printf("%s", ok ? "ok" : "fail");
            for (unsigned x = 0; x <= mask; ++x)
                if (tab[x] >= 0) std::printf(" %d", tab[x]);
            std::printf("\n");
        } else {
            return 2;
        }
    }
    return 0;
}
