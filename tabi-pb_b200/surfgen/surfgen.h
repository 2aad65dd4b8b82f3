/* surfgen.h -- MSMS-format molecular surface generator (see surfgen.c). */
#ifndef TABI_SURFGEN_H
#define TABI_SURFGEN_H
#ifdef __cplusplus
extern "C" {
#endif
/* xyzr: natm x 4 (x, y, z, radius).  On success *vert_out holds nvert x 6
 * (position, outward unit normal) and *face_out nface x 3 1-based vertex
 * indices; release both with sg_free.  blob <= 0 picks the default
 * blobbiness for the probe radius.  Returns 0, or -1 on bad arguments. */
int sg_gaussian_surface(int natm, const double* xyzr, double probe,
                        double density, double blob, double** vert_out,
                        int* nvert_out, int** face_out, int* nface_out,
                        double* spacing_out);
void sg_free(void* p);
/* Writes <prefix>.vert and <prefix>.face in the MSMS layout the reference
 * reads (readin.f90:204-246). */
int sg_write_msms(const char* prefix, int nvert, const double* vert,
                  int nface, const int* face, int natm, double density,
                  double probe);
#ifdef __cplusplus
}
#endif
#endif
