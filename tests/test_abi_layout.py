"""The ctypes mirrors of the C ABI structs have the header's layout: every
field's offset and every struct's size, read from a program that the host C
compiler builds against include/neuralsim.h (no GPU, no CUDA headers). The
oracle's config and network structs are checked the same way."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

from neuralsim_b200 import _abi as A
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = {
    "ns_config": A.NsConfig,
    "ns_drive": A.NsDrive,
    "ns_neuron_soa": A.NsNeuronSoa,
    "ns_net_desc": A.NsNetDesc,
    "ns_step_stats": A.NsStepStats,
}


ORACLE_STRUCTS = {"or_config": O.OrConfig, "or_net": O.OrNet}


def c_layout(tmp_path, header, include, structs):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include <stdint.h>',
             f'#include "{header}"', 'int main(void) {']
    for cname, cls in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ['  return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", include, str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for line in out.splitlines():
        parts = line.split()
        got[tuple(parts[:-1])] = int(parts[-1])
    return got


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a host C compiler")
@pytest.mark.parametrize("which", ["abi", "oracle"])
def test_ctypes_structs_match_the_header(tmp_path, which):
    if which == "abi":
        structs = STRUCTS
        got = c_layout(tmp_path, "neuralsim.h", os.path.join(ROOT, "include"), structs)
    else:
        structs = ORACLE_STRUCTS
        got = c_layout(tmp_path, "oracle.h", os.path.join(ROOT, "oracle"), structs)
    for cname, cls in structs.items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)
