// Test infrastructure (oracle): glibc declares newlocale and strtod_l in <locale.h> and <stdlib.h>;
// the reference includes the BSD header <xlocale.h> for them. glibc has no snprintf_l, so it is
// given here: the thread's locale is switched to the given one around vsnprintf.
#pragma once
#include <locale.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>

static inline int snprintf_l(char* buf, size_t n, locale_t loc, const char* fmt, ...) {
    locale_t old = uselocale(loc);
    va_list ap;
    va_start(ap, fmt);
    int r = vsnprintf(buf, n, fmt, ap);
    va_end(ap);
    uselocale(old);
    return r;
}
