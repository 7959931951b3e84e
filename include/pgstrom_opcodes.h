/*
 * pgstrom_opcodes.h
 *
 * Numeric values of the TypeOpCode / FuncOpCode enumerations that appear in
 * PG-Strom's kern_expression bytecode.  In the reference these enums are
 * generated from the order of src/xpu_opcodes.h (src/xpu_common.h:386-436,
 * built without WITH_POSTGIS), so the numbers are part of the wire ABI.
 * Only the opcodes this implementation translates are listed; the
 * tests (tests/test_abi.py) check every value against a table produced from
 * the reference headers (tests/golden/opcodes.txt).
 */
#ifndef PGSTROM_OPCODES_H
#define PGSTROM_OPCODES_H

/* structural opcodes (xpu_common.h:405-436) */
#define FuncOpCode__Invalid                  0
#define FuncOpCode__ConstExpr                1
#define FuncOpCode__ParamExpr                2
#define FuncOpCode__VarExpr                  3
#define FuncOpCode__BoolExpr_And             4
#define FuncOpCode__BoolExpr_Or              5
#define FuncOpCode__BoolExpr_Not             6
#define FuncOpCode__NullTestExpr_IsNull      7
#define FuncOpCode__NullTestExpr_IsNotNull   8
#define FuncOpCode__BoolTestExpr_IsTrue      9
#define FuncOpCode__BoolTestExpr_IsNotTrue   10
#define FuncOpCode__BoolTestExpr_IsFalse     11
#define FuncOpCode__BoolTestExpr_IsNotFalse  12
#define FuncOpCode__BoolTestExpr_IsUnknown   13
#define FuncOpCode__BoolTestExpr_IsNotUnknown 14
#define FuncOpCode__DistinctFrom             15
#define FuncOpCode__CoalesceExpr             16
#define FuncOpCode__LeastExpr                17
#define FuncOpCode__GreatestExpr             18
#define FuncOpCode__CaseWhenExpr             19
#define FuncOpCode__ScalarArrayOpAny         20
#define FuncOpCode__ScalarArrayOpAll         21
#define FuncOpCode__HashedArrayOp            22
#define FuncOpCode__LoadVars                 9999
#define FuncOpCode__MoveVars                 10000
#define FuncOpCode__JoinQuals                10001
#define FuncOpCode__HashValue                10002
#define FuncOpCode__GiSTEval                 10003
#define FuncOpCode__SaveExpr                 10004
#define FuncOpCode__AggFuncs                 10005
#define FuncOpCode__Projection               10006
#define FuncOpCode__SortKeys                 10007
#define FuncOpCode__Packed                   10008

/* TypeOpCode values (xpu_opcodes.h order; xpu_common.h:386-395) */
#define TypeOpCode__bool             1
#define TypeOpCode__int1             2
#define TypeOpCode__int2             3
#define TypeOpCode__int4             4
#define TypeOpCode__int8             5
#define TypeOpCode__float2           6
#define TypeOpCode__float4           7
#define TypeOpCode__float8           8
#define TypeOpCode__numeric          9
#define TypeOpCode__bytea            10
#define TypeOpCode__text             11
#define TypeOpCode__bpchar           12
#define TypeOpCode__date             13
#define TypeOpCode__time             14
#define TypeOpCode__timetz           15
#define TypeOpCode__timestamp        16
#define TypeOpCode__timestamptz      17
#define TypeOpCode__interval         18

/* FuncOpCode values used by this implementation (xpu_common.h:397-436) */
#define FuncOpCode__int2pl                   80
#define FuncOpCode__int2mi                   105
#define FuncOpCode__int2mul                  130
#define FuncOpCode__int2div                  155
#define FuncOpCode__int2eq                   206
#define FuncOpCode__int2ne                   231
#define FuncOpCode__int2lt                   281
#define FuncOpCode__int2le                   331
#define FuncOpCode__int2gt                   256
#define FuncOpCode__int2ge                   306
#define FuncOpCode__int24pl                  81
#define FuncOpCode__int24mi                  106
#define FuncOpCode__int24mul                 131
#define FuncOpCode__int24div                 156
#define FuncOpCode__int24eq                  207
#define FuncOpCode__int24ne                  232
#define FuncOpCode__int24lt                  282
#define FuncOpCode__int24le                  332
#define FuncOpCode__int24gt                  257
#define FuncOpCode__int24ge                  307
#define FuncOpCode__int28pl                  82
#define FuncOpCode__int28mi                  107
#define FuncOpCode__int28mul                 132
#define FuncOpCode__int28div                 157
#define FuncOpCode__int28eq                  208
#define FuncOpCode__int28ne                  233
#define FuncOpCode__int28lt                  283
#define FuncOpCode__int28le                  333
#define FuncOpCode__int28gt                  258
#define FuncOpCode__int28ge                  308
#define FuncOpCode__int42pl                  84
#define FuncOpCode__int42mi                  109
#define FuncOpCode__int42mul                 134
#define FuncOpCode__int42div                 159
#define FuncOpCode__int42eq                  210
#define FuncOpCode__int42ne                  235
#define FuncOpCode__int42lt                  285
#define FuncOpCode__int42le                  335
#define FuncOpCode__int42gt                  260
#define FuncOpCode__int42ge                  310
#define FuncOpCode__int4pl                   85
#define FuncOpCode__int4mi                   110
#define FuncOpCode__int4mul                  135
#define FuncOpCode__int4div                  160
#define FuncOpCode__int4eq                   211
#define FuncOpCode__int4ne                   236
#define FuncOpCode__int4lt                   286
#define FuncOpCode__int4le                   336
#define FuncOpCode__int4gt                   261
#define FuncOpCode__int4ge                   311
#define FuncOpCode__int48pl                  86
#define FuncOpCode__int48mi                  111
#define FuncOpCode__int48mul                 136
#define FuncOpCode__int48div                 161
#define FuncOpCode__int48eq                  212
#define FuncOpCode__int48ne                  237
#define FuncOpCode__int48lt                  287
#define FuncOpCode__int48le                  337
#define FuncOpCode__int48gt                  262
#define FuncOpCode__int48ge                  312
#define FuncOpCode__int82pl                  88
#define FuncOpCode__int82mi                  113
#define FuncOpCode__int82mul                 138
#define FuncOpCode__int82div                 163
#define FuncOpCode__int82eq                  214
#define FuncOpCode__int82ne                  239
#define FuncOpCode__int82lt                  289
#define FuncOpCode__int82le                  339
#define FuncOpCode__int82gt                  264
#define FuncOpCode__int82ge                  314
#define FuncOpCode__int84pl                  89
#define FuncOpCode__int84mi                  114
#define FuncOpCode__int84mul                 139
#define FuncOpCode__int84div                 164
#define FuncOpCode__int84eq                  215
#define FuncOpCode__int84ne                  240
#define FuncOpCode__int84lt                  290
#define FuncOpCode__int84le                  340
#define FuncOpCode__int84gt                  265
#define FuncOpCode__int84ge                  315
#define FuncOpCode__int8pl                   90
#define FuncOpCode__int8mi                   115
#define FuncOpCode__int8mul                  140
#define FuncOpCode__int8div                  165
#define FuncOpCode__int8eq                   216
#define FuncOpCode__int8ne                   241
#define FuncOpCode__int8lt                   291
#define FuncOpCode__int8le                   341
#define FuncOpCode__int8gt                   266
#define FuncOpCode__int8ge                   316
#define FuncOpCode__float8pl                 99
#define FuncOpCode__float8mi                 124
#define FuncOpCode__float8mul                149
#define FuncOpCode__float8div                174
#define FuncOpCode__float8eq                 225
#define FuncOpCode__float8ne                 250
#define FuncOpCode__float8lt                 300
#define FuncOpCode__float8le                 350
#define FuncOpCode__float8gt                 275
#define FuncOpCode__float8ge                 325
#define FuncOpCode__date_eq                  440
#define FuncOpCode__numeric_eq               399
#define FuncOpCode__date_ne                  441
#define FuncOpCode__numeric_ne               400
#define FuncOpCode__date_lt                  442
#define FuncOpCode__numeric_lt               401
#define FuncOpCode__date_le                  443
#define FuncOpCode__numeric_le               402
#define FuncOpCode__date_gt                  444
#define FuncOpCode__numeric_gt               403
#define FuncOpCode__date_ge                  445
#define FuncOpCode__numeric_ge               404
#define FuncOpCode__text_eq                  548
#define FuncOpCode__text_ne                  549
#define FuncOpCode__bpchareq                 541
#define FuncOpCode__int2_to_int4             37
#define FuncOpCode__int2_to_int8             43
#define FuncOpCode__int2_to_float8           61
#define FuncOpCode__float8_to_int2           35
#define FuncOpCode__int4_to_int2             31
#define FuncOpCode__int4_to_int8             44
#define FuncOpCode__int4_to_float8           62
#define FuncOpCode__float8_to_int4           41
#define FuncOpCode__int8_to_int2             32
#define FuncOpCode__int8_to_int4             38
#define FuncOpCode__int8_to_float8           63
#define FuncOpCode__float8_to_int8           47
#define FuncOpCode__int4_to_bool             23

#endif /* PGSTROM_OPCODES_H */
