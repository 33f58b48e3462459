"""The C ABI: the library loads, exports every declared symbol, and its
struct layouts match the ctypes mirror.  No GPU needed."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "hqt.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(hqt_[a-z_]+)\s*\(", text)
    return sorted(set(names))


def test_every_declared_symbol_is_exported(hqt):
    lib = hqt._lib.load()
    names = declared_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(hqt._lib.EXPORTS) == names


def test_abi_version(hqt):
    assert hqt._lib.load().hqt_abi_version() == 2


def test_struct_layout_matches_c(hqt, tmp_path):
    src = tmp_path / "layout.c"
    src.write_text("""
#include <stdio.h>
#include <stddef.h>
#include "hqt.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\\n", sizeof(hqt_params), offsetof(hqt_params, Lx),
         offsetof(hqt_params, remove_winding), offsetof(hqt_params, apply_filter),
         sizeof(hqt_diag));
  printf("%zu %zu\\n", offsetof(hqt_diag, capacity), offsetof(hqt_diag, records));
  return 0;
}
""")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    P, D = hqt._lib.hqt_params, hqt._lib.hqt_diag
    got = [ctypes.sizeof(P), P.Lx.offset, P.remove_winding.offset,
           P.apply_filter.offset, ctypes.sizeof(D), D.capacity.offset, D.records.offset]
    assert [int(v) for v in out] == got


@pytest.mark.parametrize("kw,code", [
    (dict(nx=2), 1), (dict(nz=2), 5), (dict(nz=41), 5), (dict(Lx=-1.0), 1),
    (dict(dt=float("nan")), 1),
])
def test_create_rejects_bad_parameters(hqt, kw, code):
    base = dict(nx=16, nz=9, Lx=10.0)
    base.update(kw)
    with pytest.raises(hqt.HQTError) as e:
        hqt.Simulation(**base)
    assert e.value.code == code


def test_null_context_is_rejected(hqt):
    lib = hqt._lib.load()
    assert lib.hqt_step(None, None, None, None, None, None, 1, None) == 1
    assert lib.hqt_last_error(None) is not None


def test_noalloc_rejects_misaligned_field_without_a_gpu(hqt):
    """The allocation-free count checks its arguments before any CUDA call:
    an interleaved-complex field that is not 16-byte aligned is HQT_EINVAL."""
    lib = hqt._lib.load()
    n = ctypes.c_int32()
    code = lib.hqt_count_vortices_field_noalloc(ctypes.c_void_p(0x10008), 16, 16, 8,
                                                ctypes.byref(n), ctypes.byref(n),
                                                ctypes.byref(n), None)
    assert code == 1
    assert b"aligned" in lib.hqt_noalloc_last_error()
