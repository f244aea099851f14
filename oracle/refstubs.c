/*
 * refstubs.c -- link stubs for reference functions that the background and
 * filter path of oracle/_ref never calls (TEST INFRASTRUCTURE ONLY).
 * Compiled without the reference headers so the signatures need not match.
 */
#include <stdio.h>
#include <stdlib.h>
#define STUB(name) void name(void) { fprintf(stderr, "refharness: " #name " not available\n"); abort(); }
STUB(copyimage)
STUB(pasteimage)
STUB(fitsread)
STUB(read_cat)
STUB(close_cat)
STUB(free_cat)
STUB(name_to_tab)
STUB(loadtab_bpann)
STUB(play_bpann)
STUB(free_bpann)
