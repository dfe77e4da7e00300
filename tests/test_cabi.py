"""The C-ABI library loads and exports every function include/w2w_raster.h
declares; host-only entry points behave (no GPU needed, no kernel launched)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "w2w_raster.h")
LIB = os.path.join(ROOT, "word2world_b200", "libw2w_raster.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(w2w_[A-Za-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        import importlib.util
        spec = importlib.util.spec_from_file_location("w2w_build", os.path.join(os.path.dirname(LIB), "build.py"))
        b = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(b)
        b.build_lib()
    return ctypes.CDLL(LIB)


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_host_only_entry_points(lib):
    lib.w2w_status_string.restype = ctypes.c_char_p
    assert lib.w2w_version() >= 1
    assert lib.w2w_status_string(0) == b"ok"
    assert b"invalid" in lib.w2w_status_string(1)
    for fn in ("w2w_geometry_state_bytes",):
        getattr(lib, fn).restype = ctypes.c_size_t
    lib.w2w_image_state_bytes.restype = ctypes.c_size_t
    lib.w2w_binning_state_bytes.restype = ctypes.c_size_t
    lib.w2w_sort_scratch_bytes.restype = ctypes.c_size_t
    lib.w2w_geometry_offset.restype = ctypes.c_size_t
    a, b = lib.w2w_geometry_state_bytes(1000), lib.w2w_geometry_state_bytes(2000)
    assert 0 < a < b and a % 256 == 0
    assert lib.w2w_image_state_bytes(256, 256) > 0
    assert lib.w2w_binning_state_bytes(ctypes.c_longlong(100000), 256, 256) > 100000 * 24
    for name in (b"depth", b"means2D", b"cov3D", b"conic_opacity", b"rgb", b"tiles_touched", b"offsets", b"record"):
        off = lib.w2w_geometry_offset(1000, name)
        assert off % 256 == 0 and off < a
    assert lib.w2w_geometry_offset(1000, b"nope") == ctypes.c_size_t(-1).value


def test_invalid_arguments_rejected_without_gpu(lib):
    # null settings / negative sizes are rejected before any CUDA call
    assert lib.w2w_forward_geometry(None, None, None, None, None, None, None, None, None, None) == 1
    assert lib.w2w_sort_pairs_u64(None, None, None, None, ctypes.c_longlong(-1), 0, 64, None, ctypes.c_size_t(0),
                                  None) == 1
    assert lib.w2w_sort_pairs_u64(None, None, None, None, ctypes.c_longlong(0), 0, 64, None, ctypes.c_size_t(0),
                                  None) == 0
    assert lib.w2w_scan_u32(None, None, ctypes.c_longlong(-5), 0, None, ctypes.c_size_t(0), None) == 1


def test_planned_layout_helpers(lib):
    """Host-only arithmetic of the planned forward: capacities and the layout
    count recovered from a binning state's size."""
    ll, sz = ctypes.c_longlong, ctypes.c_size_t
    lib.w2w_planned_capacity.restype = ll
    lib.w2w_planned_capacity.argtypes = [ll]
    lib.w2w_binning_layout_count.restype = ll
    lib.w2w_binning_layout_count.argtypes = [ll, sz, ctypes.c_int, ctypes.c_int]
    lib.w2w_binning_state_bytes.restype = sz
    lib.w2w_binning_state_bytes.argtypes = [ll, ctypes.c_int, ctypes.c_int]
    Q = 65536
    for R in (0, 1, 1000, 65536, 4_000_000, 5_923_615):
        C = lib.w2w_planned_capacity(R)
        assert C % Q == 0 and C >= max(Q, R + R // 4)
        assert C - Q < max(Q, R + R // 4)
        for W, H in ((256, 256), (512, 512), (800, 800)):
            exact = lib.w2w_binning_state_bytes(R, W, H)
            assert lib.w2w_binning_layout_count(R, exact, W, H) == R
            planned = lib.w2w_binning_state_bytes(C, W, H)
            assert lib.w2w_binning_layout_count(R, planned, W, H) == C
            assert lib.w2w_binning_layout_count(R, planned + 256, W, H) == -1


def test_tuning_knobs_through_the_c_abi(lib):
    """Every knob the header documents is named by the library, the autotuner
    tunes all but planned_forward, and an invalid value changes nothing."""
    lib.w2w_tune_name.restype = ctypes.c_char_p
    names = [lib.w2w_tune_name(k).decode() for k in range(lib.w2w_tune_count())]
    assert names == ["blend_warps", "backward_split", "backward_ways", "binning", "blend_queue",
                     "preprocess_blocks", "planned_forward", "blend_stage"]
    text = " ".join(re.sub(r"\n\s*\*(?!/)", " ", open(HEADER).read()).split())  # comment text, one line
    for k, n in enumerate(names):
        assert f'{k} "{n}"' in text, n  # documented with its number
    assert lib.w2w_tune_name(len(names)) == b""
    stage = names.index("blend_stage")
    before = lib.w2w_tune_get(stage)
    assert before in (0, 1)
    assert lib.w2w_tune_set(stage, 2) == -1 and lib.w2w_tune_get(stage) == before
    assert lib.w2w_tune_set(stage, 1 - before) == before and lib.w2w_tune_get(stage) == 1 - before
    assert lib.w2w_tune_set(stage, before) == 1 - before
    try:
        from word2world_b200 import autotune
    except ImportError:  # the torch extension is not built: the library part above still ran
        return
    assert set(autotune.CANDIDATES) == set(names) - {"planned_forward"}


class _Settings(ctypes.Structure):  # w2w_settings, field for field
    _fields_ = [("P", ctypes.c_int), ("degree", ctypes.c_int), ("M", ctypes.c_int), ("width", ctypes.c_int),
                ("height", ctypes.c_int), ("focal_x", ctypes.c_float), ("tan_fovx", ctypes.c_float),
                ("tan_fovy", ctypes.c_float), ("scale_modifier", ctypes.c_float), ("compat_spill", ctypes.c_int),
                ("viewmatrix", ctypes.c_void_p), ("projmatrix", ctypes.c_void_p), ("campos", ctypes.c_void_p),
                ("background", ctypes.c_void_p)]


class _GeomInfo(ctypes.Structure):
    _fields_ = [("num_rendered", ctypes.c_longlong), ("depth_min_bits", ctypes.c_uint32),
                ("depth_max_bits", ctypes.c_uint32), ("error", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


def test_planned_header_decoding(lib):
    """The host half of the planned forward: decoding the 16 header bytes the
    projection pass copies out (error word, complemented minimum and maximum
    of the depth bit patterns, instance count) and the key depth bits a view
    needs (the span of its depth patterns: the bits below their common
    prefix)."""
    import struct
    decode = lib.w2w_geometry_info_from_header
    need = lib.w2w_depth_bits_needed
    info = _GeomInfo()
    for err, lo, hi, R, status in ((0, 0x3F000000, 0x3F01FFFF, 5923615, 0), (1, 7, 7, 3, 3), (2, 1, 2, 9, 4),
                                   (3, 0, 0, 0, 4), (4, 0, 0xFFFFFFFF, 1 << 29, 0)):
        hdr = ctypes.create_string_buffer(struct.pack("<4I", err, (~lo) & 0xFFFFFFFF, hi, R), 16)
        assert decode(hdr, ctypes.byref(info)) == status, (err, status)  # timeout wins over capacity
        assert (info.error, info.depth_min_bits, info.depth_max_bits, info.num_rendered) == (err, lo, hi, R)
        assert need(ctypes.byref(info)) == (lo ^ hi).bit_length()
    assert decode(None, ctypes.byref(info)) == 1 and need(None) == -1


def test_knob_defaults_match_the_header(lib):  # the fixture builds the library when absent
    """A freshly loaded library's knob values are the defaults the header
    documents (read in a child process, so no earlier test's setting leaks)."""
    import subprocess
    import sys
    text = " ".join(re.sub(r"\n\s*\*(?!/)", " ", open(HEADER).read()).split())
    doc = text[text.index("---- launch-shape tuning"):]
    code = ("import ctypes,sys; L=ctypes.CDLL(sys.argv[1]); L.w2w_tune_name.restype=ctypes.c_char_p; "
            "print(';'.join(f'{L.w2w_tune_name(k).decode()}={L.w2w_tune_get(k)}' for k in range(L.w2w_tune_count())))")
    out = subprocess.run([sys.executable, "-c", code, LIB], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    values = dict(kv.split("=") for kv in out.stdout.strip().split(";"))
    for k, (name, v) in enumerate(values.items()):
        start = doc.index(f'{k} "{name}"')
        m = re.compile(r"default (\d+)").search(doc, start)
        assert m is not None and int(m.group(1)) == int(v), (name, v, m and m.group(0))


C_HOST = r"""
#include "w2w_raster.h"
#include <stddef.h>
#include <stdio.h>
int main(void) {
  /* the structs' layout, as an FFI binding declares it */
  fprintf(stderr, "%zu %zu %zu %zu %zu %zu\n", sizeof(w2w_settings), offsetof(w2w_settings, compat_spill),
          offsetof(w2w_settings, viewmatrix), offsetof(w2w_settings, background), sizeof(w2w_geometry_info),
          offsetof(w2w_geometry_info, reserved));
  w2w_geometry_info info = {0};
  const unsigned char hdr[16] = {0};
  if (w2w_geometry_info_from_header(hdr, &info) != W2W_OK || info.num_rendered != 0) return 2;
  printf("%d %zu %lld %d", w2w_version(), w2w_geometry_state_bytes(1000), w2w_planned_capacity(100000),
         w2w_tune_count());
  for (int k = 0; k < w2w_tune_count(); ++k) printf(" %s", w2w_tune_name(k));
  printf("\n");
  return 0;
}
"""


def test_plain_c_host_compiles_links_and_runs(lib, tmp_path):
    """The header is C99 (no C++), and a C host links the library and calls its
    host-only entry points: what a cgo / JNI / N-API shim builds on."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "host.c"
    src.write_text(C_HOST)
    exe = tmp_path / "host"
    libdir = os.path.dirname(LIB)
    r = subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.dirname(HEADER),
                        str(src), "-L", libdir, "-lw2w_raster", f"-Wl,-rpath,{libdir}", "-o", str(exe)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, (r.returncode, r.stderr)
    out = r.stdout.split()
    layout = [int(x) for x in r.stderr.split()]
    S = _Settings
    assert layout == [ctypes.sizeof(S), S.compat_spill.offset, S.viewmatrix.offset, S.background.offset,
                      ctypes.sizeof(_GeomInfo), _GeomInfo.reserved.offset]
    lib.w2w_tune_name.restype = ctypes.c_char_p
    assert int(out[0]) == lib.w2w_version() and int(out[3]) == lib.w2w_tune_count()
    assert out[4:] == [lib.w2w_tune_name(k).decode() for k in range(lib.w2w_tune_count())]
