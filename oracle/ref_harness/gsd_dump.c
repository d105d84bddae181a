/* gsd_dump.c -- test infrastructure: reads a GSD file with the reference's own reader
 * (src/gsd.c, linked unmodified by the Makefile) and prints every chunk of every frame:
 *
 *   gsd_dump <file>
 *   -> "nframes <n>" then, per frame and per chunk name present in it,
 *      "<frame> <name> <N> <M> <type> <hex bytes>"
 *
 * Exit status 1 (with the gsd error code) if the reference reader refuses the file.
 */
#include <stdio.h>
#include <stdlib.h>

#include "gsd.h"

int main(int argc, char **argv)
{
    if (argc != 2) {
        fprintf(stderr, "usage: %s file.gsd\n", argv[0]);
        return 2;
    }
    struct gsd_handle h;
    int rc = gsd_open(&h, argv[1], GSD_OPEN_READONLY);
    if (rc != GSD_SUCCESS) {
        printf("open_error %d\n", rc);
        return 1;
    }
    uint64_t nf = gsd_get_nframes(&h);
    printf("nframes %llu\n", (unsigned long long)nf);
    printf("application %s\nschema %s\nschema_version %u\ngsd_version %u\n", h.header.application,
           h.header.schema, h.header.schema_version, h.header.gsd_version);
    for (uint64_t f = 0; f < nf; f++) {
        const char *name = gsd_find_matching_chunk_name(&h, "", NULL);
        while (name) {
            const struct gsd_index_entry *e = gsd_find_chunk(&h, f, name);
            if (e) {
                size_t bytes = e->N * e->M * gsd_sizeof_type((enum gsd_type)e->type);
                unsigned char *buf = (unsigned char *)malloc(bytes ? bytes : 1);
                rc = gsd_read_chunk(&h, buf, e);
                if (rc != GSD_SUCCESS) {
                    printf("read_error %d %s\n", rc, name);
                    return 1;
                }
                printf("%llu %s %llu %u %u ", (unsigned long long)f, name, (unsigned long long)e->N, e->M,
                       (unsigned)e->type);
                for (size_t k = 0; k < bytes; k++) printf("%02x", buf[k]);
                printf("\n");
                free(buf);
            }
            name = gsd_find_matching_chunk_name(&h, "", name);
        }
    }
    gsd_close(&h);
    return 0;
}
