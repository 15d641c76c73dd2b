/* ipole_b200 command line: the reference's main (src/main.c:66-819, fast
 * light) with the pixel loop on the GPU.  Same keys, same -par / --k=v /
 * -unpol / -quench handling, same stderr summary lines, and the reference's
 * exit codes for its fatal conditions (maxnstep -10, NaN -1, bad dump -1/-3,
 * histogram request 42). */
#include <stdio.h>
#include <stdlib.h>
#include <sys/time.h>

#include "ipole_b200.h"
#include "ipole_host.h"

static double wtime(void)
{
  struct timeval tv;
  gettimeofday(&tv, NULL);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

static int exit_code(int rc)
{
  switch (rc) {
    case IPG_OK: return 0;
    case IPG_E_MAXNSTEP: return -10;
    case IPG_E_NAN: return -1;
    case IPG_E_IO: return -1;
    case IPG_E_FORMAT: return -3;
    case IPG_E_ARG: return 1;
    default: return 2;
  }
}

int main(int argc, char *argv[])
{
  fprintf(stderr, "ipole-b200 (sm_100a ray pipeline)\n\n");
  double t0 = wtime();
  ipg_params p;
  int rc = ipg_params_from_argv(&p, argc, argv);
  if (rc) return (p.histo || p.histo_polar) ? 42 : exit_code(rc);

  ipg_iharm_model m;
  rc = ipg_iharm_load(&p, &m);
  if (rc) return exit_code(rc);

  int device = 0;
  const char *dev = getenv("IPG_DEVICE");
  if (dev) device = atoi(dev);
  ipg_ctx *ctx = NULL;
  rc = ipg_create(&ctx, device, 0);
  if (rc) {
    fprintf(stderr, "could not create a CUDA context on device %d: %s\n", device, ipg_strerror(rc));
    ipg_iharm_free(&m);
    return exit_code(rc);
  }
  if (p.mixed_records) rc = ipg_set_record_precision(ctx, IPG_RECORDS_MIXED);
  if (!rc && p.fp32_step) rc = ipg_set_step_precision(ctx, IPG_STEP_FP32);
  if (!rc && p.fp32_fits) rc = ipg_set_fit_precision(ctx, IPG_FITS_FP32);
  if (!rc) rc = ipg_upload_model(ctx, &m);
  if (rc) {
    fprintf(stderr, "model upload failed: %s (%s)\n", ipg_strerror(rc), ipg_last_error(ctx));
    ipg_destroy(ctx);
    ipg_iharm_free(&m);
    return exit_code(rc);
  }
  double t_init = wtime() - t0;

  ipg_image img;
  rc = ipg_render_image(ctx, &p, &m, &img, stderr);
  if (rc == IPG_OK && p.trace && !p.perform_check) {
    rc = ipg_write_traces(ctx, &img, &p, &m);
    if (rc) fprintf(stderr, "trace output failed: %s (%s)\n", ipg_strerror(rc), ipg_last_error(ctx));
  }
  if (rc == IPG_OK) {
    ipg_print_image_stats(&img, &p, stderr);
    if (!p.quench_output && p.perform_check) {
      rc = ipg_write_check(p.outf, &img, &p);
    } else if (!p.quench_output) {
      if (ipg_write_image(p.outf, &img, &p, &m) != IPG_OK) {
        fprintf(stderr, "could not write image file '%s'\n", p.outf);
        rc = IPG_E_IO;
      }
    }
  }
  ipg_image_free(&img);
  ipg_destroy(ctx);
  ipg_iharm_free(&m);
  fprintf(stderr, "Total wallclock time: %g s (%g s)\n\n", wtime() - t0, t_init);
  return exit_code(rc);
}
