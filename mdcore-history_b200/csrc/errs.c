/* Error stack of the engine API (stands in for src/errs.c:33-111 of the reference).
 *
 * Every failing API call pushes {id, message, line, function, file}; errs_dump prints the
 * stack bottom-up in the reference's "file:func:line: msg (id)" format and clears it. */
#include <stdio.h>
#include "mdcore_b200.h"

typedef struct {
    int id, line;
    const char *msg, *func, *file;
} err_entry;

static err_entry err_stack[errs_maxstack];
static int err_top = 0;

int errs_register(int id, const char *msg, int line, const char *func, const char *file) {
    if (err_top < errs_maxstack) {
        err_entry *en = &err_stack[err_top++];
        en->id = id;
        en->msg = msg;
        en->line = line;
        en->func = func;
        en->file = file;
    }
    return id;
}

void errs_clear(void) { err_top = 0; }

int errs_dump(FILE *out) {
    for (int k = 0; k < err_top; k++)
        fprintf(out, "%s:%s:%i: %s (%i)\n", err_stack[k].file, err_stack[k].func,
                err_stack[k].line, err_stack[k].msg, err_stack[k].id);
    errs_clear();
    return 0;
}
