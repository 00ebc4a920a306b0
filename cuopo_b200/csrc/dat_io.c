/*
 * dat_io.c -- the reference's .dat text format (src/headers/files.cuh:21-62):
 * one value per line written with 20 significant digits (std::setprecision(20)
 * on a float, i.e. the shortest "%.20g" form); complex vectors are split
 * into <prefix>_r.dat and <prefix>_i.dat.
 */
#include <errno.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "cuopo.h"
#include "internal.h"

static cuopo_status write_strided(const char *path, const float *v, long n, long stride)
{
    FILE *fp = fopen(path, "w");
    if (!fp) return cuopo_fail(CUOPO_EIO, "write_dat: cannot open file for writing");
    /* a large stdio buffer: these files reach N*NRT lines */
    static __thread char buf[1 << 16];
    setvbuf(fp, buf, _IOFBF, sizeof(buf));
    for (long i = 0; i < n; i++) {
        if (fprintf(fp, "%.20g\n", (double)v[i * stride]) < 0) {
            fclose(fp);
            return cuopo_fail(CUOPO_EIO, "write_dat: write failed");
        }
    }
    if (fclose(fp) != 0) return cuopo_fail(CUOPO_EIO, "write_dat: close failed");
    return CUOPO_OK;
}

cuopo_status cuopo_write_dat_real(const char *path, const float *v, long n)
{
    if (!path || (!v && n > 0) || n < 0) return cuopo_fail(CUOPO_EINVAL, "write_dat_real: bad argument");
    return write_strided(path, v, n, 1);
}

cuopo_status cuopo_write_dat_complex(const char *prefix, const float *v, long n)
{
    if (!prefix || (!v && n > 0) || n < 0) return cuopo_fail(CUOPO_EINVAL, "write_dat_complex: bad argument");
    const size_t L = strlen(prefix) + 8;
    char *path = (char *)malloc(L);
    if (!path) return cuopo_fail(CUOPO_ENOMEM, "write_dat_complex: out of memory");
    snprintf(path, L, "%s_r.dat", prefix);
    cuopo_status st = write_strided(path, v, n, 2);
    if (st == CUOPO_OK) {
        snprintf(path, L, "%s_i.dat", prefix);
        st = write_strided(path, v + 1, n, 2);
    }
    free(path);
    return st;
}

static cuopo_status read_strided(const char *path, float *v, long n, long stride)
{
    FILE *fp = fopen(path, "r");
    if (!fp) return cuopo_fail(CUOPO_EIO, "read_dat: cannot open file");
    for (long i = 0; i < n; i++) {
        double x;
        if (fscanf(fp, "%lf", &x) != 1) {
            fclose(fp);
            return cuopo_fail(CUOPO_EIO, "read_dat: file shorter than expected");
        }
        v[i * stride] = (float)x;
    }
    fclose(fp);
    return CUOPO_OK;
}

cuopo_status cuopo_read_dat_complex(const char *prefix, float *v, long n)
{
    if (!prefix || (!v && n > 0) || n < 0) return cuopo_fail(CUOPO_EINVAL, "read_dat_complex: bad argument");
    const size_t L = strlen(prefix) + 8;
    char *path = (char *)malloc(L);
    if (!path) return cuopo_fail(CUOPO_ENOMEM, "read_dat_complex: out of memory");
    snprintf(path, L, "%s_r.dat", prefix);
    cuopo_status st = read_strided(path, v, n, 2);
    if (st == CUOPO_OK) {
        snprintf(path, L, "%s_i.dat", prefix);
        st = read_strided(path, v + 1, n, 2);
    }
    free(path);
    return st;
}
