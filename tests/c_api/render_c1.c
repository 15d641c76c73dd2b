/* A C caller of the library through its installed headers only: renders an
 * image with the reference's parameters and writes it, then loads the same
 * dump through the reference's model interface (model.h names) and prints
 * a few point queries.  Built and run by tests/test_gpu_c_api.py.
 *
 *   render_c1 OUT.ipgc --dump=... [ipole keys]
 */
#include <stdio.h>
#include <stdlib.h>

#include "ipole_b200.h"
#include "ipole_host.h"

int main(int argc, char **argv)
{
  if (argc < 3) {
    fprintf(stderr, "usage: %s OUT [ipole keys]\n", argv[0]);
    return 2;
  }
  const char *out = argv[1];
  ipg_params p;
  /* argv[1] stands in for the program name of load_par_from_argv */
  int rc = ipg_params_from_argv(&p, argc - 1, argv + 1);
  ipg_iharm_model m;
  if (!rc) rc = ipg_iharm_load(&p, &m);
  if (rc) {
    fprintf(stderr, "load: %s\n", ipg_strerror(rc));
    return 3;
  }
  ipg_ctx *ctx = NULL;
  rc = ipg_create(&ctx, 0, 0);
  if (!rc) rc = ipg_upload_model(ctx, &m);
  ipg_image img;
  if (!rc) rc = ipg_render_image(ctx, &p, &m, &img, stderr);
  if (!rc) rc = ipg_write_image(out, &img, &p, &m);
  if (rc) {
    fprintf(stderr, "render: %s (%s)\n", ipg_strerror(rc), ctx ? ipg_last_error(ctx) : "");
    return 4;
  }
  double tot[5];
  ipg_image_totals(&img, &p, tot);
  printf("Ftot %.17g Ftot_unpol %.17g traced %zu\n", tot[0], tot[1], img.traced);
  ipg_image_free(&img);
  ipg_destroy(ctx);

  /* the reference's model interface on the same keys */
  if (ipg_params_from_argv(ipg_model_params(), argc - 1, argv + 1)) return 5;
  double tA = 0., tB = 0.;
  init_model(&tA, &tB);
  if (ipg_model_status()) return 6;
  const ipg_iharm_model *lm = ipg_model_loaded();
  /* the centre of zone (i, j, k) = (n1/2, n2/2, n3/2) */
  const ipg_grid *g = &lm->grid;
  int i = g->n1 / 2, j = g->n2 / 2, k = g->n3 / 2;
  double X[4] = {0., g->startx[1] + (i + 0.5) * g->dx[1], g->startx[2] + (j + 0.5) * g->dx[2],
                 g->startx[3] + (k + 0.5) * g->dx[3]};
  size_t c = ((size_t)(i + 1) * (g->n2 + 2) + (j + 1)) * (g->n3 + 2) + (k + 1);
  double K[4] = {1., 0., 0., 0.}, Ucon[4], Ucov[4], Bcon[4], Bcov[4];
  get_model_fourv(X, K, Ucon, Ucov, Bcon, Bcov);
  double udotu = Ucon[0] * Ucov[0] + Ucon[1] * Ucov[1] + Ucon[2] * Ucov[2] + Ucon[3] * Ucov[3];
  printf("M_unit %.17g t %.17g ne %.17g ne_cell %.17g thetae %.17g thetae_cell %.17g b %.17g b_cell %.17g "
         "udotu %.17g radiating %d sigma_cell %.17g\n",
         M_unit, tA, get_model_ne(X), lm->fields[IPG_F_NE][c], get_model_thetae(X), lm->fields[IPG_F_THETAE][c],
         get_model_b(X), lm->fields[IPG_F_B][c], udotu, radiating_region(X), lm->fields[IPG_F_SIGMA][c]);
  ipg_iharm_free(&m);
  return 0;
}
