"""ABI pins: struct layouts and opcode numbers equal the reference's."""
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def test_struct_layout_matches_reference(tmp_path):
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=gnu11", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "abi_layout_probe.c"), "-o", str(exe)], check=True)
    mine = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    with open(os.path.join(GOLDEN, "abi_layout.txt")) as f:
        ref = f.read()
    assert mine.splitlines() == ref.splitlines()


def test_opcodes_match_reference():
    ref = {}
    with open(os.path.join(GOLDEN, "opcodes.txt")) as f:
        for line in f:
            kind, name, val = line.split()
            ref[("FuncOpCode__" if kind == "func" else "TypeOpCode__") + name] = int(val)
    n = 0
    with open(os.path.join(ROOT, "include", "pgstrom_opcodes.h")) as f:
        for line in f:
            m = re.match(r"#define\s+((?:Func|Type)OpCode__\w+)\s+(\d+)", line)
            if not m:
                continue
            name, val = m.group(1), int(m.group(2))
            if name in ref:
                assert ref[name] == val, name
                n += 1
            else:
                # structural opcodes defined before the generated ones
                assert name.startswith("FuncOpCode__"), name
    assert n > 100
