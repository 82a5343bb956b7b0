/*
 * tslb_io.h -- output formats and checkpoints of the TSLB driver.
 *
 * The writers produce the files the reference's print_module.f90 writes, so
 * its post-processing (compare.f90, raw2vti*, ParaView) reads them unchanged:
 *
 *   tslb_write_raw     print_raw_sync (print_module.f90:679-698): a field as
 *                      unformatted stream, FP32, Fortran order, no header
 *   tslb_write_vti     print_vtk_sync / print_vtk_phionly_sync (:899-929)
 *                      with the header of header_vtk/footer_vtk (:9-214):
 *                      VTK ImageData, WholeExtent "1 nx 1 ny 1 nz", one
 *                      Float32 DataArray (1 or 3 components) in raw appended
 *                      form: header, '_', int32 byte count, data, footer
 *   tslb_write_slices  print_raw_slice_2c_sync (:812-897): the mid planes
 *                      f(:,:,nz/2), f(:,ny/2,:), f(nx/2,:,:) (1-based
 *                      halves) as <dir>/out_<name>xy|xz|yz_<frame>.raw
 *   tslb_frame_path    <dir>/<prefix>_<name>_<frame>.<ext> with the frame
 *                      zero-padded to 6 digits (write_fmtnumb, :511-544)
 *
 * Checkpoints replace dump_distros_1c_3d / read_distros_1c_3d (:700-723):
 * the reference dumps its populations; here the state is the 11 moment
 * fields, saved in their storage type (bit-exact for every precision)
 * with the storage scales, the parameters and the step counter.  The
 * inlet planes, the tau correction and an attached closure are the
 * driver's and are not part of a checkpoint.
 *
 * The writers are host code and need no GPU.  Every function returns
 * TSLB_OK or TSLB_ERR_ARG (bad argument or I/O failure) / TSLB_ERR_CUDA.
 */
#ifndef TSLB_IO_H
#define TSLB_IO_H

#include "tslb.h"

#ifdef __cplusplus
extern "C" {
#endif

int tslb_write_raw(const char* path, const float* data, long long n);
/* name: up to 8 characters (blank-padded as the reference's namevar);
 * ncomp 1 (scalar, nx*ny*nz values) or 3 (vector, components fastest). */
int tslb_write_vti(const char* path, const char* name, int nx, int ny, int nz, int ncomp, const float* data);
int tslb_write_slices(const char* dir, const char* name, int frame, int nx, int ny, int nz, const float* field);
int tslb_frame_path(char* out, int cap, const char* dir, const char* prefix, const char* name, int frame,
                    const char* ext);

int tslb_checkpoint_save(tslb_ctx* ctx, const char* path);
/* The lattice must have the sizes, mode and precision of the file. */
int tslb_checkpoint_load(tslb_ctx* ctx, const char* path);
/* Step counter of the context (steps advanced since creation or since the
 * loaded checkpoint's save). */
long long tslb_steps_done(tslb_ctx* ctx);

/* Page-locked host memory for the upload and download arrays of a host that
 * does not call the CUDA runtime itself (a Fortran driver, tslb_run): copies
 * from and to it run at the full PCIe rate without a staging copy.  No
 * counterpart in the reference, whose arrays are plain Fortran allocations.
 * tslb_host_alloc returns NULL on failure; tslb_host_free(NULL) does nothing. */
void* tslb_host_alloc(long long bytes);
void  tslb_host_free(void* p);

#ifdef __cplusplus
}
#endif

#endif /* TSLB_IO_H */
