"""The C ABI from a C program: include/cupami_b200.h compiles as C (gcc, -std=c99
-Wall -Werror), links against libcupami_b200.so, and the host-only entry points
(version, default options, pattern trees and their ordering) run without a GPU."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]

C_SOURCE = r"""
#include <stdio.h>
#include <string.h>
#include "cupami_b200.h"

int main(void) {
    cpm_opts o;
    if (cpm_default_opts(&o) != CPM_OK) return 1;
    printf("%s\n", cpm_version());
    /* patterns {0}, {1}, {0,1}, {2}, {1,2} as a tree emitted out of order */
    const int64_t parent[5] = {-1, -1, 1, -1, 0};
    const uint32_t item[5] = {1, 0, 1, 2, 2};
    const uint64_t support[5] = {7, 9, 5, 4, 3};
    cpm_result *res = NULL;
    if (cpm_result_from_tree(parent, item, support, 5, &res) != CPM_OK) return 2;
    uint64_t n = 0, slots = 0;
    if (cpm_result_size(res, &n, &slots) != CPM_OK || n != 5 || slots != 7) return 3;
    uint64_t offsets[6], sup[5];
    uint32_t items[7];
    if (cpm_result_copy(res, CPM_ORDER_APRIORI, offsets, items, sup) != CPM_OK) return 4;
    for (uint64_t k = 0; k < n; ++k) {
        printf("[");
        for (uint64_t i = offsets[k]; i < offsets[k + 1]; ++i) printf(i > offsets[k] ? " %u" : "%u", items[i]);
        printf("]:%llu\n", (unsigned long long)sup[k]);
    }
    int64_t periods[5];
    /* a frequent-itemset result has no periodicities */
    if (cpm_result_copy_periodic(res, CPM_ORDER_APRIORI, offsets, items, sup, periods) != CPM_EINVAL) return 5;
    cpm_result_free(res);
    return 0;
}
"""


def test_header_compiles_as_c_and_host_calls_run(tmp_path):
    from cupami_b200 import _native

    lib = _native.LIB_PATH
    if not lib.exists():
        pytest.skip("library not built")
    src = tmp_path / "caller.c"
    src.write_text(C_SOURCE)
    exe = tmp_path / "caller"
    subprocess.check_call(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"),
                           str(src), "-o", str(exe), "-L", str(lib.parent), "-lcupami_b200",
                           f"-Wl,-rpath,{lib.parent}"])
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.splitlines()
    assert lines[0].startswith("cupami_b200")
    # by length, then tuple (the Apriori order): {0}, {1}, {2}, {0,1}, {1,2}
    assert lines[1:] == ["[0]:9", "[1]:7", "[2]:4", "[0 1]:5", "[1 2]:3"]
