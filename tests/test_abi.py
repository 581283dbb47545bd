"""CPU tests of the C ABI boundary: the library loads, exports every symbol
include/harmony_b200.h declares, and fails cleanly without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import harmony_b200 as hb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "harmony_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_api():
    syms = declared_symbols()
    for s in ("hb_create", "hb_train", "hb_add", "hb_search", "hb_save_index", "hb_load_index",
              "hb_set_nprobe", "hb_last_error"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    L = hb.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_params_defaults():
    L = hb.lib()
    p = hb._SearchParamsC()
    L.hb_search_params_init(ctypes.byref(p))
    assert p.mode == hb.SearchMode.ORIGINAL
    assert p.order_optimize == 1 and p.pruning == 0
    assert p.warmup_lists == 10 and p.warmup_list_size == 0
    assert p.precision == hb.Precision.FP32


def test_enums_match_reference_values():
    # src/common.h:20-37, src/Index.h:29-35
    assert int(hb.MetricType.METRIC_L2) == 1 and int(hb.MetricType.METRIC_IP) == 0
    assert [int(m) for m in hb.SearchMode] == [0, 1, 2, 3, 4]
    assert int(hb.OptLevel.OPT_ALL) == 7


def test_null_handle_is_an_error():
    L = hb.lib()
    assert L.hb_train(None, 0, None, 0) == 1
    assert b"null index handle" in L.hb_last_error()
    assert L.hb_destroy(None) == 0


def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(hb.HarmonyError) as e:
        hb.Index(8, 4, 2)
    assert e.value.code == 6  # HB_ERR_NODEVICE


def test_struct_layout_matches_header(tmp_path):
    """ctypes mirror of hb_search_params has the C compiler's layout."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "%s"\n'
                   'int main(){printf("%%zu %%zu %%zu", sizeof(hb_search_params),'
                   ' offsetof(hb_search_params, nprobe_per_query), offsetof(hb_search_params, max_nprobe));}'
                   % HEADER)
    exe = tmp_path / "sz"
    subprocess.check_call([cc, str(src), "-o", str(exe)])
    size, off_ptr, off_max = map(int, subprocess.check_output([str(exe)]).split())
    S = hb._SearchParamsC
    assert (ctypes.sizeof(S), S.nprobe_per_query.offset, S.max_nprobe.offset) == (size, off_ptr, off_max)


def test_cpp_dropin_header_compiles_and_links(tmp_path):
    """A driver written against the reference's harmony::Index compiles against
    include/harmony_b200_index.hpp and links libharmony_b200.so."""
    import shutil
    import subprocess
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "driver.cpp"
    src.write_text(r'''
#include "harmony_b200_index.hpp"
#include <cstdio>
#include <vector>
int main() {
  try {
    harmony::Index index(8, 4, 2, harmony::METRIC_L2, harmony::OPT_NONE, 0, 1, 1, false);
    std::vector<float> x(64 * 8, 1.0f);
    index.train(64, x.data());
    index.add(64, x.data());
    harmony::Index::Param p;
    p.mode = harmony::Index::SearchMode::ORIGINAL;
    index.preSearch(64, 0, 0, 0, 0, &p, "");
    std::vector<float> D(2 * 3);
    std::vector<harmony::idx_t> I(2 * 3);
    index.search(2, x.data(), 3, D.data(), I.data());
    std::printf("ok %ld\n", (long)I[0]);
  } catch (const std::exception& e) {
    std::printf("error %s\n", e.what());
  }
  return 0;
}
''')
    exe = tmp_path / "driver"
    subprocess.check_call([cxx, "-std=c++17", str(src), "-I", os.path.join(ROOT, "include"),
                           "-L", os.path.dirname(hb.LIB_PATH), "-lharmony_b200",
                           "-Wl,-rpath," + os.path.dirname(hb.LIB_PATH), "-o", str(exe)])
    out = subprocess.check_output([str(exe)]).decode()
    import torch
    if torch.cuda.is_available():
        assert out.startswith("ok")
    else:
        assert "no CUDA device" in out
