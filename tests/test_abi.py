"""The C-ABI libraries load on a CPU-only machine and export every entry point that
include/*.h declares (no compute call is made here)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "chfem_b200", "lib")


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = [n for n in re.findall(r"\b((?:cudapcg|hmg|chfemB200|cudapcgB200)\w*)\s*\(", text) if not n.endswith("_t")]
    return sorted(set(names))


@pytest.mark.parametrize("header,lib", [("cudapcg_b200.h", "libcudapcg_b200.so"), ("chfem_b200.h", "libchfem_b200.so")])
def test_exports(header, lib):
    path = os.path.join(LIB, lib)
    assert os.path.exists(path), f"{path} not built"
    handle = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)
    names = declared(header)
    assert len(names) > 20 if header == "cudapcg_b200.h" else len(names) > 25
    missing = [n for n in names if not hasattr(handle, n)]
    assert not missing, f"{lib} lacks {missing}"


def test_cli_help():
    import subprocess
    p = subprocess.run([os.path.join(LIB, "chfem_exec"), "-h"], capture_output=True, text=True, timeout=60)
    assert p.returncode == 0 and "-pm" in p.stdout and "--precision" in p.stdout


def test_errors_are_reported_not_fatal(tmp_path):
    """A bad input returns an error code and message; the process survives (no exit())."""
    from chfem_b200 import _native
    lib = _native.chfem()
    lib.chfemB200SetQuiet(1)
    nf = tmp_path / "bad.nf"
    nf.write_text("%type_of_analysis\n0\n%image_dimensions\n4 4 0\n%number_of_materials\n1\n%properties_of_materials\n0 1.0\n")
    raw = tmp_path / "bad.raw"
    raw.write_bytes(bytes(16))
    sdf = str(tmp_path / "field.bin").encode()
    assert lib.hmgInit(str(nf).encode(), str(raw).encode(), sdf, None) == 0  # density field file missing
    assert b"field.bin" in lib.chfemB200LastError()
    # 2D with more than 16 materials for 16-bit keys of 4 bits per pixel
    mats = "".join(f"{i} {i + 1}\n" for i in range(17))
    nf.write_text(f"%type_of_analysis\n0\n%image_dimensions\n4 4 0\n%number_of_materials\n17\n%properties_of_materials\n{mats}")
    raw.write_bytes(bytes([i % 17 for i in range(16)]))
    assert lib.hmgInit(str(nf).encode(), str(raw).encode(), None, None) == 0
    assert b"16 materials" in lib.chfemB200LastError()
    # truncated image
    nf.write_text("%type_of_analysis\n0\n%image_dimensions\n4 4 4\n%number_of_materials\n1\n%properties_of_materials\n0 1.0\n")
    assert lib.hmgInit(str(nf).encode(), str(raw).encode(), None, None) == 0
    assert b"end of image" in lib.chfemB200LastError()
    # colour not listed in the .nf
    raw.write_bytes(bytes([0] * 63 + [7]))
    assert lib.hmgInit(str(nf).encode(), str(raw).encode(), None, None) == 0
    assert b"colour 7" in lib.chfemB200LastError()
    # more than 4 materials for 16-bit keys
    nf.write_text("%type_of_analysis\n0\n%image_dimensions\n4 4 4\n%number_of_materials\n5\n%properties_of_materials\n0 1\n1 2\n2 3\n3 4\n4 5\n")
    raw.write_bytes(bytes([i % 5 for i in range(64)]))
    assert lib.hmgInit(str(nf).encode(), str(raw).encode(), None, None) == 0
    assert b"4 materials" in lib.chfemB200LastError()


def test_cudapcg_rejects_out_of_scope():
    from chfem_b200 import _native
    lib = _native.cudapcg()
    assert lib.cudapcgInit(6, 0) == 0            # no such analysis
    assert b"invalid analysis" in lib.cudapcgB200LastError()
    assert lib.cudapcgInit(4, 1) == 0            # 2D Stokes with EBE
    assert lib.cudapcgInit(5, 1) == 0            # Stokes with EBE


def test_batch_input_errors():
    """compute_conductivity_batch rejects bad input before any GPU work."""
    import numpy as np
    from chfem_b200 import compute_conductivity_batch
    img = np.zeros((4, 4, 4), np.uint8)
    img[0, 0, 0] = 7
    with pytest.raises(ValueError):
        compute_conductivity_batch([img], {0: 1.0})            # colour 7 has no conductivity
    with pytest.raises(ValueError):
        compute_conductivity_batch([img], [{0: 1.0}, {0: 2.0}])  # one dict per image
    with pytest.raises(ValueError):
        compute_conductivity_batch([np.zeros((4, 4), np.uint8)], {0: 1.0})
    with pytest.raises(ValueError):
        compute_conductivity_batch([img], {0: 1.0, 7: 2.0}, precision="fp16")
