/* Built and run by tests/test_c_abi_from_c.py: the header compiles as C99 and
 * a C host links the library and gets status codes without a GPU (the mesh
 * checks of crimson_ctx_create run on the host before any device work). */
#include <stdio.h>
#include <string.h>

#include "crimson_b200.h"

int main(void) {
    crimson_params p;
    memset(&p, 0, sizeof(p));
    p.rho = 1.06;
    p.mu = 0.04;
    p.alfi = 1.0;
    p.almi = 1.5;
    p.gami = 1.0;
    p.Delt = 1e-3;
    p.Dtgl = 1e3;
    p.dtsfct = 1.0;
    p.taucfct = 1.0;
    p.idiff = 1;
    p.iconvflow = 2;
    p.ibksiz = 255;
    p.ndofBC = 7;
    p.nthreads = 1;
    /* one tet, column-major x (4, 3) and ien (1, 4), 1-based; flat (zero volume) */
    double x[12] = {0, 1, 0, 0.5, /* x */ 0, 0, 1, 0.5, /* y */ 0, 0, 0, 0 /* z */};
    int ien[4] = {1, 2, 3, 4};
    crimson_ctx* ctx = NULL;
    int rc = crimson_ctx_create(&ctx, &p, 4, 4, 1, ien, x);
    printf("version=%s rc=%d msg=%s\n", crimson_version(), rc, crimson_last_error());
    return (rc == CRIMSON_ERR_ARG && ctx == NULL) ? 0 : 1;
}
