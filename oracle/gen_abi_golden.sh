#!/bin/sh
# Regenerates the ABI pins under tests/golden/ from the reference headers.
# Reads PG-Strom's src/ directory, given as $PGSTROM_SRC (required); run it
# only where that tree exists.  Outputs:
#   tests/golden/abi_layout.txt  sizeof/offsetof of every ABI field used
#   tests/golden/opcodes.txt     TypeOpCode / FuncOpCode name -> value
set -e
SRC=${PGSTROM_SRC:?set PGSTROM_SRC to the PG-Strom src/ directory}
HERE=$(cd "$(dirname "$0")/.." && pwd)
TMP=$(mktemp -d)
gcc -std=gnu11 -DUSE_REFERENCE -I"$SRC" "$HERE/tests/abi_layout_probe.c" -o "$TMP/layout"
"$TMP/layout" > "$HERE/tests/golden/abi_layout.txt"
cat > "$TMP/ops.c" <<'XEOF'
#include <stdio.h>
#define CUDA_MAXTHREADS_PER_BLOCK 512
#include "xpu_common.h"
int main(void)
{
#define TYPE_OPCODE(NAME,a,b) printf("type %s %d\n", #NAME, (int)TypeOpCode__##NAME);
#include "xpu_opcodes.h"
#undef TYPE_OPCODE
#define TYPE_OPCODE(NAME,a,b)
#define FUNC_OPCODE(a,b,c,NAME,d,e) printf("func %s %d\n", #NAME, (int)FuncOpCode__##NAME);
#define DEVONLY_FUNC_OPCODE(a,NAME,b,c,d) printf("func %s %d\n", #NAME, (int)FuncOpCode__##NAME);
#include "xpu_opcodes.h"
    printf("func LoadVars %d\nfunc HashValue %d\nfunc SaveExpr %d\nfunc Packed %d\n",
           (int)FuncOpCode__LoadVars, (int)FuncOpCode__HashValue,
           (int)FuncOpCode__SaveExpr, (int)FuncOpCode__Packed);
    return 0;
}
XEOF
gcc -std=gnu11 -I"$SRC" "$TMP/ops.c" -o "$TMP/ops"
"$TMP/ops" > "$HERE/tests/golden/opcodes.txt"
rm -rf "$TMP"
echo "wrote tests/golden/abi_layout.txt tests/golden/opcodes.txt"
