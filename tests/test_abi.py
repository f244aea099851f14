"""The C ABI library loads and exports every entry point of include/sexgpu.h;
the ctypes layouts match the C structs (CPU only: no compute calls)."""
import os
import re
import subprocess
import tempfile

import pytest

import sexgpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "sexgpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char \*)\s*\**\s*(sexgpu_\w+)\s*\(", src, re.M)))


def test_library_exports_header_symbols():
    lib = sexgpu.lib()
    names = header_functions()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(sexgpu.EXPORTS)


def test_struct_layouts_match_header():
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "sexgpu.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(sexgpu_config), sizeof(sexgpu_object),
         offsetof(sexgpu_object, mx), offsetof(sexgpu_object, poserr_mx2),
         offsetof(sexgpu_object, polar), sizeof(sexgpu_summary), sizeof(sexgpu_stage));
  return 0;
}'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(prog)
        exe = os.path.join(d, "t")
        subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe])
        vals = [int(v) for v in subprocess.check_output([exe]).split()]
    import ctypes as C
    dt = sexgpu.OBJECT_DTYPE
    assert vals == [C.sizeof(sexgpu.Config), dt.itemsize, dt.fields["mx"][1], dt.fields["poserr_mx2"][1],
                    dt.fields["polar"][1], C.sizeof(sexgpu.Summary), C.sizeof(sexgpu.Stage)]


def test_config_rejected_without_device_work():
    """Argument errors are reported as status codes (no GPU needed)."""
    import ctypes as C
    lib = sexgpu.lib()
    assert lib.sexgpu_create(None, 0) == -1
    assert lib.sexgpu_destroy(None) == -1


COMPAT_NAMES = ["init_device", "clear_device", "back_estimate", "cudaFilter", "init_detection", "run_detection",
                "clear_detection", "init_deblend", "parcel_out", "clear_deblend", "analyse_gpu", "run_clean",
                "endobject_gpu", "sexgpu_compat_configure", "sexgpu_compat_set_device", "sexgpu_compat_set_nnw",
                "sexgpu_compat_set_error_handler"]


def test_compat_library_exports_reference_names():
    """libsexgpu_compat.so exports the thirteen entry points of the reference's
    src/cuda/*.h (and libsexgpu.so none of them)."""
    import ctypes as C
    path = os.path.join(ROOT, "gpu-sextractor_b200", "libsexgpu_compat.so")
    lib = C.CDLL(path)
    for n in COMPAT_NAMES:
        assert hasattr(lib, n), n
    src = open(os.path.join(ROOT, "include", "sexgpu_compat.h")).read()
    declared = set(re.findall(r"^(?:int|void)\s+(\w+)\s*\(", src, re.M))
    assert declared == set(COMPAT_NAMES)
    main = sexgpu.lib()
    assert not hasattr(main, "init_device") and not hasattr(main, "parcel_out")


def test_compat_record_layout():
    """sexgpu_outobj has the member offsets of the reference's outobjstruct
    (src/types.h:417-455 with NAPER = 1, 16-byte aligned)."""
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "sexgpu_compat.h"
#define O(m) (int)offsetof(sexgpu_outobj, m)
int main(void) {
  printf("%d %d %d %d %d %d %d %d %d %d %d %d\n", (int)sizeof(sexgpu_outobj), O(alpha2000), O(sposx),
         O(flux_aper), O(magerr_aper), O(theta), O(poserr_mx2), O(poserr_mxy), O(flag), O(elong), O(sprob), O(fwhm));
  return 0;
}'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(prog)
        exe = os.path.join(d, "t")
        subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe])
        vals = [int(v) for v in subprocess.check_output([exe]).split()]
    assert vals == [160, 8, 24, 56, 68, 88, 96, 112, 120, 124, 132, 148]


def test_batch_frame_layout():
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "sexgpu.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(sexgpu_batch_frame), offsetof(sexgpu_batch_frame, objs),
         offsetof(sexgpu_batch_frame, status), offsetof(sexgpu_batch_frame, summary));
  return 0;
}'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(prog)
        exe = os.path.join(d, "t")
        subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe])
        vals = [int(v) for v in subprocess.check_output([exe]).split()]
    import ctypes as C
    B = sexgpu.BatchFrame
    assert vals == [C.sizeof(B), B.objs.offset, B.status.offset, B.summary.offset]


def test_read_nnw(tmp_path):
    """sexgpu_read_nnw parses the .nnw layout (host code, no GPU needed)."""
    import pytest
    import sexgpu
    from conftest import synthetic_nnw, write_nnw
    net = synthetic_nnw(3)
    path = tmp_path / "t.nnw"
    write_nnw(str(path), net)
    got = sexgpu.read_nnw(str(path))
    nn, inbias, inscale, weights, biases, outbias, outscale = net
    assert got.nlayers == 3 and list(got.nn) == nn
    assert list(got.inbias) == list(inbias) and list(got.inscale) == list(inscale)
    for l in range(2):
        for j in range(nn[l + 1]):
            assert got.b[l][j] == biases[l][j]
            for i in range(nn[l]):
                assert got.w[l][i][j] == weights[l][i][j]
    assert got.outbias[0] == outbias[0] and got.outscale[0] == outscale[0]
    bad = tmp_path / "bad.nnw"
    bad.write_text("not a network\n1 2 3\n")
    with pytest.raises(RuntimeError):
        sexgpu.read_nnw(str(bad))


OUTOBJ_MEMBERS = ["number", "alpha2000", "delta2000", "sposx", "sposy", "flux_iso", "fluxerr_iso", "mag_iso",
                  "magerr_iso", "flux_isocor", "fluxerr_isocor", "flux_aper", "fluxerr_aper", "mag_aper",
                  "magerr_aper", "flux_auto", "fluxerr_auto", "mag_auto", "magerr_auto", "theta", "poserr_mx2",
                  "poserr_my2", "poserr_mxy", "flag", "elong", "ellip", "sprob", "peak", "kronfactor", "bkg",
                  "fwhm"]


def test_compat_record_layout_matches_reference_header():
    """sizeof and every member offset of sexgpu_outobj equal those of the
    reference's own outobjstruct (src/types.h:417-455), compiled from its
    header into oracle/_ref; skipped where the reference tree is absent."""
    import ctypes as C
    from oracle import oracle as O
    r = O.ref()
    if r is None:
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    buf = (C.c_int * 64)()
    n = r.ref_outobj_layout(buf, 64)
    ref = list(buf[:n])
    prog = "#include <stdio.h>\n#include <stddef.h>\n#include \"sexgpu_compat.h\"\nint main(void){printf(\"%d" + \
        " %d" * len(OUTOBJ_MEMBERS) + "\\n\", (int)sizeof(sexgpu_outobj)" + \
        "".join(", (int)offsetof(sexgpu_outobj, %s)" % m for m in OUTOBJ_MEMBERS) + ");return 0;}\n"
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(prog)
        exe = os.path.join(d, "t")
        subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe])
        ours = [int(v) for v in subprocess.check_output([exe]).split()]
    assert n == 1 + len(OUTOBJ_MEMBERS)
    assert ours == ref
