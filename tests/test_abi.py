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


def test_c_client_of_the_abi(tmp_path):
    """include/xpu_b200.h compiles as strict C99 and the library links into
    a C program (PG-Strom's GPU service is C); from C, xpuB200HashBytes
    equals the reference's pg_hash_any on its committed vectors, and
    xpuB200Init attaches GPU 0 or, without one, fails with an error code
    and a message rather than crashing."""
    import json
    lib_dir = os.path.join(ROOT, "pg-strom_b200")
    if not os.path.exists(os.path.join(lib_dir, "libxpu_b200.so")):
        import pytest
        pytest.skip("library not built")
    exe = tmp_path / "abi_c_client"
    subprocess.run(["gcc", "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror",
                    "-I" + os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "abi_c_client.c"),
                    "-L" + lib_dir, "-lxpu_b200", "-Wl,-rpath," + lib_dir, "-o", str(exe)], check=True)
    with open(os.path.join(GOLDEN, "ref_scalars.json")) as f:
        vec = json.load(f)["hash_any"]
    stdin = "\n".join(f"{h or '-'} {v}" for h, v in vec) + "\n"
    r = subprocess.run([str(exe)], input=stdin, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    lines, bad, init = r.stdout.split()
    assert (int(lines), int(bad)) == (len(vec), 0)
    assert init in ("ok", "error")
