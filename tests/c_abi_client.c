/* A plain C (C99) client of libdg_b200.so: what a binding from another
 * language (cgo, JNI, N-API, ctypes) sees. Host-only calls, no GPU: Gauss
 * tables, the periodic box generator (sizes first, then arrays), the
 * reference's HDF5 mesh reader, the variant tables, and the error convention
 * (status codes, dg_last_error(NULL) for calls without a context).
 * Usage: c_abi_client <quad_1x1.h5>; prints "ok" and exits 0 on success. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dg_b200.h"

#define CHECK(cond)                                                         \
    do {                                                                    \
        if (!(cond)) {                                                      \
            fprintf(stderr, "check failed at line %d: %s\n", __LINE__, #cond); \
            return 1;                                                       \
        }                                                                   \
    } while (0)

int main(int argc, char** argv)
{
    double x[5], w[5], s = 0.0;
    int i;
    CHECK(argc == 2);
    CHECK(dg_gauss_legendre(5, x, w) == DG_OK);
    for (i = 0; i < 5; ++i) s += w[i];
    CHECK(fabs(s - 2.0) < 1e-14);
    CHECK(fabs(x[2]) < 1e-15);

    {
        const int n[3] = {2, 3, 4};
        const double x0[3] = {0.0, 0.0, 0.0}, len[3] = {1.0, 1.0, 1.0};
        int nnode = 0, nelem = 0, nface = 0;
        double* coords;
        unsigned *e2n, *faces;
        CHECK(dg_mesh_periodic_box(n, x0, len, 7u, &nnode, NULL, &nelem, NULL, &nface, NULL) == DG_OK);
        CHECK(nelem == 24 && nface == 72 && nnode == 3 * 4 * 5);
        coords = malloc(sizeof(double) * 3 * (size_t)nnode);
        e2n = malloc(sizeof(unsigned) * 8 * (size_t)nelem);
        faces = malloc(sizeof(unsigned) * 8 * (size_t)nface);
        CHECK(coords && e2n && faces);
        CHECK(dg_mesh_periodic_box(n, x0, len, 7u, &nnode, coords, &nelem, e2n, &nface, faces) == DG_OK);
        for (i = 0; i < 8 * nelem; ++i) CHECK(e2n[i] < (unsigned)nnode);
        free(coords);
        free(e2n);
        free(faces);
    }

    {
        int dim = 0, q = 0, npe = 0, nnode = 0, nelem = 0, nface = 0;
        CHECK(dg_mesh_read_h5(argv[1], &dim, &q, &npe, &nnode, NULL, &nelem, NULL, &nface, NULL) == DG_OK);
        CHECK(dim == 2 && q == 1 && npe == 4 && nelem == 1 && nface == 2);
        CHECK(dg_mesh_read_h5("/nonexistent/mesh.h5", &dim, &q, &npe, &nnode, NULL, &nelem, NULL, &nface, NULL) ==
              DG_ERR_ARG);
        CHECK(strstr(dg_last_error(NULL), "cannot open") != NULL);
    }

    {
        int nv = dg_num_stage_variants(3), E = 0, NT = 0, G = 0, prec = -1;
        CHECK(nv > 0);
        CHECK(dg_stage_variant_info(3, 0, &E, &NT, &G, &prec) == DG_OK);
        CHECK(E >= 1 && NT >= 32 && NT % 32 == 0 && (prec == 0 || prec == 1));
    }

    CHECK(dg_probe_bounded_wait(0, -1, 0, NULL) == DG_ERR_ARG);
    CHECK(strlen(dg_last_error(NULL)) > 0);
    printf("ok\n");
    return 0;
}
