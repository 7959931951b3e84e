/*
 * abi_c_client.c -- a plain C99 client of the C ABI, built and run by
 * tests/test_abi.py: include/xpu_b200.h compiles as C (PG-Strom's GPU
 * service is C), the library links into a C program, and calls that need
 * no GPU behave as documented.
 *
 * stdin: lines "<hex bytes or -> <hash>" (PG-Strom's pg_hash_any of the
 * bytes, computed by the reference's own function).  Checks
 * xpuB200HashBytes against every line, then that xpuB200Init either
 * attaches GPU 0 (and shuts it down again) or fails with an error code and
 * a message.  Prints "<lines> <mismatches> <init: ok|error>"; exits 1 on any
 * mismatch or on a failure without a message.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "xpu_b200.h"

static int hexval(char c)
{
    if (c >= '0' && c <= '9') return c - '0';
    if (c >= 'a' && c <= 'f') return c - 'a' + 10;
    return -1;
}

int main(void)
{
    static char hex[4096];
    static unsigned char buf[2048];
    unsigned long want;
    int lines = 0, bad = 0;
    xpuB200Device *dev = NULL;
    kern_errorbuf err;
    int rc;

    while (scanf("%4095s %lu", hex, &want) == 2) {
        size_t len = strcmp(hex, "-") == 0 ? 0 : strlen(hex) / 2;
        size_t i;
        uint32_t got;

        if (len > sizeof(buf))
            return 2;
        for (i = 0; i < len; i++) {
            int hi = hexval(hex[2 * i]), lo = hexval(hex[2 * i + 1]);
            if (hi < 0 || lo < 0)
                return 2;
            buf[i] = (unsigned char)(hi * 16 + lo);
        }
        got = xpuB200HashBytes(buf, (uint32_t)len);
        if (got != (uint32_t)want) {
            fprintf(stderr, "length %lu: %u, want %lu\n", (unsigned long)len, got, want);
            bad++;
        }
        lines++;
    }

    memset(&err, 0, sizeof(err));
    rc = xpuB200Init(0, 0, &dev, &err);
    if (rc == 0) {
        xpuB200Shutdown(dev);
        printf("%d %d ok\n", lines, bad);
    } else {
        if (err.errcode == 0 || err.message[0] == '\0')
            return 1;
        fprintf(stderr, "init: %s\n", err.message);
        printf("%d %d error\n", lines, bad);
    }
    return bad ? 1 : 0;
}
