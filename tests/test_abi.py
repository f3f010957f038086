"""The C ABI library on CPU (no GPU calls): it loads, exports every function
that include/*.h declares, and the ctypes struct layouts of the bindings
match the compiler's sizeof()."""
import ctypes as C
import os
import re
import subprocess

from shape_b200 import ctypes_defs as cd
from shape_b200 import engine as eng

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("shape_b200.h", "shape_types.h"):
        text = open(os.path.join(REPO, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(shape_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_loads_and_exports_all_declared_symbols():
    L = eng.load_library()
    assert L.shape_version().startswith(b"shape-b200")
    names = declared_functions()
    assert "shape_engine_evaluate" in names and "shape_chi2_frames_noalloc" in names
    out = subprocess.run(["nm", "-D", "--defined-only", eng.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = sorted(n for n in names if n not in exported)
    assert not missing, missing
    for n in names:
        assert hasattr(L, n)


def test_struct_layouts_match_compiler():
    sizes = eng.abi_sizes()
    for name, size in zip(eng.ABI_ORDER, sizes):
        assert C.sizeof(cd.STRUCTS[name]) == size, name
    assert C.sizeof(eng.EvalSummary) == sizes[len(eng.ABI_ORDER)]
    for k, name in enumerate(("shape_doppler_frame", "shape_doppler_set")):
        assert C.sizeof(cd.STRUCTS[name]) == sizes[len(eng.ABI_ORDER) + 1 + k], name
    assert C.sizeof(cd.SpinState) == sizes[len(eng.ABI_ORDER) + 3], "shape_spin_state"
    assert C.sizeof(cd.EphemPoint) == sizes[len(eng.ABI_ORDER) + 4], "shape_ephem_point"
    assert C.sizeof(cd.PosetFrame) == sizes[len(eng.ABI_ORDER) + 5], "shape_poset_frame"
    assert C.sizeof(cd.PosetSet) == sizes[len(eng.ABI_ORDER) + 6], "shape_poset_set"
    assert C.sizeof(cd.PosetResult) == sizes[len(eng.ABI_ORDER) + 7], "shape_poset_result"


def test_errors_without_device_are_reported():
    """Without a usable device, create fails with a status and a message
    (the library never falls back to a CPU path)."""
    import torch
    if torch.cuda.is_available():
        return
    L = eng.load_library()
    h = C.c_void_p()
    rc = L.shape_engine_create(0, C.byref(h))
    assert rc < 0 and len(L.shape_last_error()) > 0


def test_dropin_compiles_against_reference_headers(tmp_path):
    """The calc_fits drop-in compiles against the reference's struct
    definitions and exports calc_fits (signature of src/shape/shape2.h:1451)
    and calc_fits_chi2_b200 under their default names."""
    import pytest
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    ref_src = os.environ.get("REF_ROOT", os.path.join(os.path.dirname(repo), "reference")) + "/src"
    if not os.path.isdir(os.path.join(ref_src, "shape")):
        pytest.skip("reference headers not present")
    inc = ["-I" + os.path.join(ref_src, d) for d in ("shape", "util", "nr", "astro", "pgm",
                                                     "HostMultiThreading")]
    obj = str(tmp_path / "dropin.o")
    subprocess.run(["gcc", "-O2", "-std=gnu99", "-w", "-c", "-iquote",
                    os.path.join(repo, "oracle", "refshim", "shape"), "-I-",
                    "-I" + os.path.join(repo, "oracle", "refshim", "shape")] + inc +
                   ["-I/usr/local/cuda/include", "-I" + os.path.join(repo, "include"),
                    "-I" + os.path.join(repo, "shape-cuda-v1.2_b200", "dropin"),
                    os.path.join(repo, "shape-cuda-v1.2_b200", "dropin", "shape_b200_dropin.c"), "-o", obj],
                   check=True)
    syms = subprocess.run(["nm", "-g", "--defined-only", obj], capture_output=True, text=True,
                          check=True).stdout.split()
    assert "calc_fits" in syms and "calc_fits_chi2_b200" in syms
