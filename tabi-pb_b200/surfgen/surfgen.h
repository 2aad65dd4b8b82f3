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
/* Random sequential addition over a stream of candidate points (ncand x 3,
 * scanned in order): takes candidates inside the ball of `radius` that keep
 * distance >= min_sep to every point placed so far, until natm are placed.
 * pts (natm x 3) holds *placed points on entry, which are kept.  Returns the
 * number of candidates consumed (-1 on bad arguments). */
int sg_rsa(int natm, double radius, double min_sep, const double* cand, int ncand,
           double* pts, int* placed);
/* Writes <prefix>.vert and <prefix>.face in the MSMS layout the reference
 * reads (readin.f90:204-246). */
int sg_write_msms(const char* prefix, int nvert, const double* vert,
                  int nface, const int* face, int natm, double density,
                  double probe);
#ifdef __cplusplus
}
#endif
#endif
