/* abi_harness.c -- calls librgf_b200.so through include/rgf.h exactly as the
 * Fortran ISO_C_BINDING interface does: scalars by reference, column-major
 * complex(8) arrays, int64 dimensions, optional arguments as NULL.
 *
 *   abi_harness layout            print struct sizes / offsets
 *   abi_harness nogpu             context creation must fail cleanly without a GPU
 *   abi_harness solve IN OUT      one green_RGF_RS call; IN/OUT are raw binaries
 *   abi_harness solve_rgfg IN OUT the same through RGF_G's argument order
 *
 * IN:  int64 nm, nx, has_sigma; double E, mu[2], temp[2];
 *      c16 Hii[nm*nm*nx], H1i[...]; if has_sigma: c16 sig_lesser[...], sig_r[...]
 * OUT: double tr, tre; c16 ndens, pdens, ldos, GRi1 [nm*nm*nx]; double cur[nm*nm*nx]
 */
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "rgf.h"

static int rd(FILE* f, void* p, size_t n) { return fread(p, 1, n, f) == n ? 0 : -1; }

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  if (!strcmp(argv[1], "layout")) {
    printf("opts %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(rgf_opts),
           offsetof(rgf_opts, eta_dev), offsetof(rgf_opts, eta_lead), offsetof(rgf_opts, boltz),
           offsetof(rgf_opts, sancho_tol), offsetof(rgf_opts, sancho_nmax),
           offsetof(rgf_opts, consistent), offsetof(rgf_opts, precision),
           offsetof(rgf_opts, want_T), offsetof(rgf_opts, verbose), offsetof(rgf_opts, reserved));
    printf("device %zu %zu %zu %zu %zu\n", sizeof(rgf_device), offsetof(rgf_device, Hii),
           offsetof(rgf_device, mu), offsetof(rgf_device, temp), offsetof(rgf_device, Sii));
    printf("task %zu %zu %zu %zu %zu\n", sizeof(rgf_task), offsetof(rgf_task, E),
           offsetof(rgf_task, sigma_lesser), offsetof(rgf_task, cur), offsetof(rgf_task, T));
    printf("info %zu\n", sizeof(rgf_task_info));
    printf("c16 %zu\n", sizeof(rgf_c16));
    return 0;
  }
  if (!strcmp(argv[1], "nogpu")) {
    rgf_opts o;
    rgf_opts_default(&o);
    rgf_ctx* c = NULL;
    int rc = rgf_ctx_create(&o, &c);
    printf("%d %s|%s\n", rc, rgf_version(), rgf_last_error());
    if (c) rgf_ctx_destroy(c);
    return 0;
  }
  if ((!strcmp(argv[1], "solve") || !strcmp(argv[1], "solve_rgfg")) && argc == 4) {
    FILE* f = fopen(argv[2], "rb");
    if (!f) return 3;
    int64_t nm, nx, has_sig;
    double E, mu[2], temp[2];
    if (rd(f, &nm, 8) || rd(f, &nx, 8) || rd(f, &has_sig, 8) || rd(f, &E, 8) || rd(f, mu, 16) ||
        rd(f, temp, 16))
      return 4;
    const size_t n = (size_t)nm * nm * nx;
    rgf_c16* Hii = malloc(n * sizeof(rgf_c16));
    rgf_c16* H1i = malloc(n * sizeof(rgf_c16));
    rgf_c16* sl = NULL;
    rgf_c16* sr = NULL;
    if (rd(f, Hii, n * 16) || rd(f, H1i, n * 16)) return 5;
    if (has_sig) {
      sl = malloc(n * 16);
      sr = malloc(n * 16);
      if (rd(f, sl, n * 16) || rd(f, sr, n * 16)) return 6;
    }
    fclose(f);
    rgf_c16* nd = calloc(n, 16);
    rgf_c16* pd = calloc(n, 16);
    rgf_c16* ld = calloc(n, 16);
    rgf_c16* gr = calloc(n, 16);
    double* cur = calloc(n, 8);
    double tr = 0, tre = 0;
    int rc;
    if (!strcmp(argv[1], "solve"))
      rc = rgf_green_rgf_rs(NULL, temp, &nm, &nx, &E, mu, Hii, H1i, sl, NULL, sr, nd, pd, ld, &tr,
                            &tre, cur, gr, NULL, NULL);
    else
      rc = rgf_rgf_g(NULL, temp, &nm, &nx, &E, mu, Hii, H1i, sl, NULL, sr, &tr, &tre, nd, pd, ld,
                     cur, gr, NULL, NULL);
    if (rc != RGF_OK) {
      fprintf(stderr, "rc=%d %s\n", rc, rgf_last_error());
      return 7;
    }
    FILE* g = fopen(argv[3], "wb");
    fwrite(&tr, 8, 1, g);
    fwrite(&tre, 8, 1, g);
    fwrite(nd, 16, n, g);
    fwrite(pd, 16, n, g);
    fwrite(ld, 16, n, g);
    fwrite(gr, 16, n, g);
    fwrite(cur, 8, n, g);
    fclose(g);
    return 0;
  }
  return 2;
}
