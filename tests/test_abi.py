"""The C ABI library loads, exports every entry point its header declares, and
its structs have the same layout in C and in the ctypes binding (no GPU)."""
import ctypes
import re
import subprocess
import textwrap
from pathlib import Path

import pytest

from feelmri_b200 import _lib as L

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "feelmri_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^FM_API\s+\w+\s+(fm_\w+)\(", text, flags=re.M)))


def test_library_built_and_loads():
    lib = L.lib()
    assert lib.fm_abi_version() == 1


def test_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 19
    lib = L.lib()
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert set(syms) == set(L.SIGNATURES), "ctypes signatures and header declarations differ"


def test_errors_without_device_are_reported_not_thrown():
    lib = L.lib()
    assert lib.fm_ctx_destroy(None) == L.FM_ERR_ARG
    assert "null fm_ctx" in L.last_error()
    nbytes = ctypes.c_size_t()
    assert lib.fm_signal_workspace_size(None, 0, ctypes.byref(nbytes)) == L.FM_ERR_ARG


def test_count_time_runs_host_helper():
    import numpy as np
    from feelmri_b200 import ops
    t = np.array([1, 1, 2, 2, 2, 1, np.nan, np.nan, 3], np.float32)
    # NaN never equals itself, so each NaN starts a run (MRI.cpp:109)
    assert ops.count_time_runs(t) == 6
    assert ops.count_time_runs(t.astype(np.float64)) == 6
    assert ops.count_time_runs(np.zeros(0, np.float32)) == 0


STRUCTS = {
    "fm_motion_term": (L.MotionTerm, ["kind", "modes", "pp_c", "pp_x", "pp_k", "timeshift", "period", "direction",
                                      "extrapolate"]),
    "fm_motion": (L.Motion, ["kind", "n_terms", "terms", "table", "table_calls"]),
    "fm_bloch_args": (L.BlochArgs, ["n_pos", "r0", "M0", "gamma", "rf", "motion", "Mz_final", "Mxy_carry",
                                    "final_stride"]),
    "fm_signal_args": (L.SignalArgs, ["n_nodes", "m_nnz", "m_data", "kx", "Mxy", "motion", "out"]),
    "fm_mass_args": (L.MassArgs, ["n_elems", "nodes_per_elem", "elems", "n_qpoints", "tabulated"]),
    "fm_tc_tuning": (L.TcTuning, ["split_nodes", "kz_cap", "reserved"]),
    "fm_bloch_block": (L.BlochBlock, ["offset", "n_time", "empty", "store", "timeshift", "timeshift_kind"]),
    "fm_bloch_sequence_args": (L.BlochSequenceArgs, ["n_pos", "M0", "gamma", "n_blocks", "blocks", "n_samples",
                                                     "rf", "motion", "n_store", "Mxy_out", "Mz_carry"]),
}


def test_struct_layouts_match_header(tmp_path):
    lines = []
    for cname, (_, fields) in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in fields:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    src = textwrap.dedent("""
        #include <stdio.h>
        #include <stddef.h>
        #include "feelmri_b200.h"
        int main(void) {
        %s
        return 0; }
    """) % "\n".join(lines)
    c = tmp_path / "probe.c"
    c.write_text(src)
    exe = tmp_path / "probe"
    gcc = "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc"
    r = subprocess.run([gcc, "-I", str(ROOT / "include"), str(c), "-o", str(exe)], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail(r.stderr)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    for line in out:
        if not line:
            continue
        cname, what, val = line.split()
        klass = STRUCTS[cname][0]
        if what == "size":
            assert ctypes.sizeof(klass) == int(val), (cname, what)
        else:
            assert getattr(klass, what).offset == int(val), (cname, what)
