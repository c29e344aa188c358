"""The ctypes mirrors of the C-ABI structs (lambda_vm_b200/native.py) against
include/starkgpu.h as a C compiler lays them out: every struct's size and
every field's offset, from a C program compiled with plain gcc (no GPU)."""
import ctypes as C
import os
import subprocess

from lambda_vm_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PAIRS = [("LeafLayout", "sg_leaf_layout"), ("TableDesc", "sg_table_desc"), ("PassRecord", "sg_pass_record"),
         ("Rv64Info", "sg_rv64_info"), ("VerifyTable", "sg_verify_table"), ("LdeInfo", "sg_lde_info"),
         ("DeviceProgram", "sg_device_program"), ("Composition", "sg_composition"), ("LogupDesc", "sg_logup_desc"),
         ("TableJob", "sg_table_job"), ("ProofShape", "sg_proof_shape"), ("TableProof", "sg_table_proof")]


def test_ctypes_structs_match_the_header(tmp_path):
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "starkgpu.h"', "int main(void) {"]
    for py, c in PAIRS:
        lines.append(f'    printf("{py} size %zu\\n", sizeof({c}));')
        for name, _ in getattr(native, py)._fields_:
            lines.append(f'    printf("{py} {name} %zu\\n", offsetof({c}, {name}));')
    lines += ["    return 0;", "}"]
    src, exe = tmp_path / "layout.c", tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    r = subprocess.run(["gcc", "-std=c11", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for py, _ in PAIRS:
        cls = getattr(native, py)
        assert got[(py, "size")] == C.sizeof(cls), py
        for name, _ in cls._fields_:
            assert got[(py, name)] == getattr(cls, name).offset, (py, name)
