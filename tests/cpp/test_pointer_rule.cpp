// Host-only check of the rule cfdb_solve_device_noalloc applies to the caller's arrays
// (cfd_b200/csrc/pointer_rule.hpp): device memory of the current device or managed memory.
#include "pointer_rule.hpp"

#include <cstdio>

int main() {
    using namespace cfdb;
    int fails = 0;
    auto expect = [&](bool got, bool want, const char* what) {
        if (got != want) {
            std::printf("FAIL %s\n", what);
            ++fails;
        }
    };
    expect(pointer_usable_on(kPtrDevice, 0, 0), true, "device memory of the current device");
    expect(pointer_usable_on(kPtrDevice, 1, 0), false, "device memory of another device");
    expect(pointer_usable_on(kPtrDevice, 0, 3), false, "device 0 memory while device 3 is current");
    expect(pointer_usable_on(kPtrManaged, 2, 0), true, "managed memory");
    expect(pointer_usable_on(kPtrHost, 0, 0), false, "page-locked host memory");
    expect(pointer_usable_on(kPtrUnregistered, -2, 0), false, "pageable host memory");
    if (fails == 0) std::printf("ok\n");
    return fails == 0 ? 0 : 1;
}
