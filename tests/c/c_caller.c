/* A plain C99 caller of the sorter's C ABI, the way the reference's C++
 * sorter or any other host program would bind it: formats two host records
 * as spike lines and asks for a handle with an empty configuration (refused
 * with a status code and a message, no GPU needed). */
#include <stdint.h>
#include <stdio.h>

#include "lss.h"

int main(void) {
    int64_t t[2] = {100, 250};
    int32_t y[2] = {3, 0};
    float a[2] = {12.5f, 0.25f};
    lss_records r = {0};
    r.time = t;
    r.template_id = y;
    r.amplitude = a;
    r.capacity = 2;
    r.count = 2;
    r.on_device = 0;
    char buf[256];
    const int64_t n = lss_format_spike_lines(&r, 1000, 0, buf, (int64_t)sizeof buf);
    if (n < 0) {
        fprintf(stderr, "%s\n", lss_last_error(0));
        return 1;
    }
    fputs(buf, stdout);
    lss_config c = {0};
    lss_handle* h = 0;
    const int rc = lss_create(&c, 0, &h);
    printf("create=%d handle=%s error=%s\n", rc, h ? "set" : "null", lss_last_error(0)[0] ? "yes" : "no");
    return 0;
}
