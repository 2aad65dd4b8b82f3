/*
 * tabi_msms -- command-line front end of surfgen.c with the flags the
 * reference passes to MSMS (readin.f90:201):
 *     tabi_msms -if <file>.xyzr -prob 1.4 -de <density> -of <prefix> [-blob B]
 * Reads "x y z r" lines, writes <prefix>.vert and <prefix>.face.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "surfgen.h"

int main(int argc, char** argv) {
  const char *in = NULL, *out = NULL;
  double probe = 1.4, den = 1.0, blob = 0.0;
  for (int i = 1; i + 1 < argc; i += 2) {
    if (!strcmp(argv[i], "-if")) in = argv[i + 1];
    else if (!strcmp(argv[i], "-of")) out = argv[i + 1];
    else if (!strcmp(argv[i], "-prob")) probe = atof(argv[i + 1]);
    else if (!strcmp(argv[i], "-de")) den = atof(argv[i + 1]);
    else if (!strcmp(argv[i], "-blob")) blob = atof(argv[i + 1]);
    else {
      fprintf(stderr, "tabi_msms: unknown flag %s\n", argv[i]);
      return 2;
    }
  }
  if (!in || !out) {
    fprintf(stderr, "usage: tabi_msms -if f.xyzr -prob 1.4 -de den -of prefix [-blob B]\n");
    return 2;
  }
  FILE* f = fopen(in, "r");
  if (!f) {
    fprintf(stderr, "tabi_msms: cannot open %s\n", in);
    return 1;
  }
  int cap = 1024, n = 0;
  double* xyzr = (double*)malloc(sizeof(double) * 4 * cap);
  double a, b, c, r;
  while (fscanf(f, "%lf %lf %lf %lf", &a, &b, &c, &r) == 4) {
    if (n == cap) {
      cap *= 2;
      xyzr = (double*)realloc(xyzr, sizeof(double) * 4 * cap);
    }
    xyzr[4 * n] = a;
    xyzr[4 * n + 1] = b;
    xyzr[4 * n + 2] = c;
    xyzr[4 * n + 3] = r;
    n++;
  }
  fclose(f);
  double *vert;
  int *face, nv, nf;
  double h;
  if (sg_gaussian_surface(n, xyzr, probe, den, blob, &vert, &nv, &face, &nf, &h)) {
    fprintf(stderr, "tabi_msms: surface generation failed\n");
    return 1;
  }
  if (sg_write_msms(out, nv, vert, nf, face, n, den, probe)) {
    fprintf(stderr, "tabi_msms: cannot write %s.vert/.face\n", out);
    return 1;
  }
  printf("tabi_msms: %d atoms -> %d vertices, %d faces (grid %.3f A)\n", n, nv, nf, h);
  sg_free(vert);
  sg_free(face);
  free(xyzr);
  return 0;
}
