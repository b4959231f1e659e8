/* Drop-in replacement for the reference's cudasymmfft/funcinterface.h:
 * identical C++-linkage signatures (funcinterface.h:5-32), so code written
 * against libcudasymmfft.a links against libcuhelmholtz_b200.so unchanged.
 *
 * Behaviour kept from the reference: device pointers, the padded
 * (NZ+2)(NY+2)(NX+2) [z][y][x] layout, synchronous return, and process exit
 * with the reference's message on an in-place call with a non-cubic grid
 * (funcinterface.cu:27-33).  The stream-ordered, status-returning form is
 * chz_do_transform in cuhelmholtz_b200.h. */
#ifndef __FUNC_INTERFACE__
#define __FUNC_INTERFACE__
#include "global.h"

/* funcinterface.h:5-12 */
void do_transform(double *d_data,
                  double *d_out,
                  int NX,
                  int NY,
                  int NZ,
                  transform_kind X_TRANS,
                  transform_kind Y_TRANS,
                  transform_kind Z_TRANS);

/* funcinterface.h:14-21 -- out-of-place; d_data is left unchanged. */
void do_transform_nocubic(double *d_data,
                          double *d_out,
                          int NX,
                          int NY,
                          int NZ,
                          transform_kind X_TRANS,
                          transform_kind Y_TRANS,
                          transform_kind Z_TRANS);

/* funcinterface.h:23-29 -- in place. */
void do_transform_cubic(double *d_data,
                        int NX,
                        int NY,
                        int NZ,
                        transform_kind X_TRANS,
                        transform_kind Y_TRANS,
                        transform_kind Z_TRANS);

/* funcinterface.h:32 -- the reference destroys its per-call cuFFT plans here;
 * this build keeps no per-call state, so it is a no-op. */
void freeMemory_cubic();
#endif /* __FUNC_INTERFACE__ */
