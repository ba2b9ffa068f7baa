/* A Cedar C-API program (the calls of include/cedar/capi.h) run against
 * libcdrgpu.so: 2D five- or nine-point Poisson entered vertex by vertex with
 * cedar_mat_set2d, a solve with cedar_solver_run and the residual by
 * cedar_matvec.  Usage: cedar_poisson config.json n stencil(5|9) out.bin
 * Writes the solution and then the right-hand side it solved with (each
 * ghost-inclusive, (n+2)^2 doubles) to out.bin and prints the relative
 * residual. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "cedar_capi.h"

#define CHECK(call)                                                        \
	do {                                                                   \
		int e_ = (call);                                                   \
		if (e_ != CEDAR_SUCCESS) {                                         \
			fprintf(stderr, "%s failed: %d\n", #call, e_);                 \
			return 10 + e_;                                                \
		}                                                                  \
	} while (0)

int main(int argc, char **argv)
{
	if (argc < 5) return 2;
	const unsigned n = (unsigned)atoi(argv[2]);
	const int nine = atoi(argv[3]) == 9;
	cedar_config conf;
	cedar_topo topo;
	cedar_mat mat;
	cedar_vec x, b, y;
	cedar_solver slv;
	CHECK(cedar_config_create(argv[1], &conf));
	CHECK(cedar_log_init(conf));
	unsigned lnx[1] = {n}, lny[1] = {n};
	CHECK(cedar_topo_create2d(0, n, n, lnx, lny, 1, 1, &topo));
	CHECK(cedar_mat_create2d(conf, topo, nine ? CEDAR_STENCIL_NINE_PT : CEDAR_STENCIL_FIVE_PT, &mat));
	/* vertex-based rows of the matrix: 5-pt 4/-1, 9-pt (bilinear FE) 8/-1 */
	const double h = 1.0 / (n + 1);
	for (unsigned j = 0; j < n; ++j)
		for (unsigned i = 0; i < n; ++i) {
			cedar_coord_2d c[9];
			cedar_real v[9];
			unsigned k = 0;
			c[k].i = i; c[k].j = j; c[k].dir = BMG2_C; v[k++] = nine ? 8.0 : 4.0;
			if (i > 0) { c[k].i = i; c[k].j = j; c[k].dir = BMG2_W; v[k++] = -1.0; }
			if (j > 0) { c[k].i = i; c[k].j = j; c[k].dir = BMG2_S; v[k++] = -1.0; }
			if (i + 1 < n) { c[k].i = i; c[k].j = j; c[k].dir = BMG2_E; v[k++] = -1.0; }
			if (j + 1 < n) { c[k].i = i; c[k].j = j; c[k].dir = BMG2_N; v[k++] = -1.0; }
			if (nine) {
				if (i > 0 && j > 0) { c[k].i = i; c[k].j = j; c[k].dir = BMG2_SW; v[k++] = -1.0; }
				if (i + 1 < n && j > 0) { c[k].i = i; c[k].j = j; c[k].dir = BMG2_SE; v[k++] = -1.0; }
				if (i + 1 < n && j + 1 < n) { c[k].i = i; c[k].j = j; c[k].dir = BMG2_NE; v[k++] = -1.0; }
				if (i > 0 && j + 1 < n) { c[k].i = i; c[k].j = j; c[k].dir = BMG2_NW; v[k++] = -1.0; }
			}
			CHECK(cedar_mat_set2d(mat, k, c, v));
		}
	CHECK(cedar_vec_create2d(topo, &x));
	CHECK(cedar_vec_create2d(topo, &b));
	CHECK(cedar_vec_create2d(topo, &y));
	cedar_real *xb, *bb, *yb;
	cedar_len ilen, jlen;
	CHECK(cedar_vec_baseptr(x, &xb));
	CHECK(cedar_vec_baseptr(b, &bb));
	CHECK(cedar_vec_baseptr(y, &yb));
	CHECK(cedar_vec_len2d(b, &ilen, &jlen));
	if (ilen != n + 2 || jlen != n + 2) return 3;
	const double pi = 3.14159265358979323846;
	for (unsigned j = 1; j <= n; ++j)
		for (unsigned i = 1; i <= n; ++i)
			bb[j * ilen + i] = 8 * pi * pi * sin(2 * pi * i * h) * sin(2 * pi * j * h) * h * h;
	CHECK(cedar_solver_create(mat, &slv));
	CHECK(cedar_solver_run(slv, x, b));
	CHECK(cedar_matvec(mat, x, y));
	double rr = 0, bn = 0;
	for (unsigned j = 1; j <= n; ++j)
		for (unsigned i = 1; i <= n; ++i) {
			const double r = bb[j * ilen + i] - yb[j * ilen + i];
			rr += r * r;
			bn += bb[j * ilen + i] * bb[j * ilen + i];
		}
	printf("relative residual %.6e\n", sqrt(rr / bn));
	FILE *f = fopen(argv[4], "wb");
	if (!f) return 4;
	fwrite(xb, sizeof(double), (size_t)ilen * jlen, f);
	fwrite(bb, sizeof(double), (size_t)ilen * jlen, f);
	fclose(f);
	CHECK(cedar_solver_destroy(&slv));
	CHECK(cedar_vec_free(&x));
	CHECK(cedar_vec_free(&b));
	CHECK(cedar_vec_free(&y));
	CHECK(cedar_mat_free(&mat));
	CHECK(cedar_topo_free(&topo));
	CHECK(cedar_config_free(&conf));
	return 0;
}
