/* nessi_io.h — libcntr's plain-text herm_matrix format for checkpoint and restart.
 *
 * Host-side C ABI of nessi_b200/libnessi_io.so (no CUDA).  Arrays are host buffers in libcntr's
 * herm_matrix layout (cntr_herm_matrix_impl.hpp:457-477): ret and les packed triangles of
 * (nt+1)(nt+2)/2 elements, tv (nt+1)(ntau+1) elements with tau fastest, mat ntau+1 elements;
 * an element is size1 x size1 complex doubles, row-major.  A device batch is checkpointed by
 * downloading G (nessi_gpu_get_G) and printing it, and restarted by reading the time steps up to
 * nt1 and uploading them (nessi_gpu_set_G) before stepping on from nt1 + 1.
 *
 * Every function returns 0 on success, 1 (NESSI_ERR_ARG) on a bad argument, an unreadable or
 * malformed file; nessi_io_last_error() describes the failure.  libcntr aborts the process on a
 * malformed file (cntr_herm_matrix_impl.hpp:1383-1386); here the caller gets the error.
 */
#ifndef NESSI_IO_H
#define NESSI_IO_H

#ifdef __cplusplus
extern "C" {
#endif

const char *nessi_io_last_error(void);

/* herm_matrix::print_to_file(file, precision) (cntr_herm_matrix_decl.hpp:166,
 * cntr_herm_matrix_impl.hpp:1308-1361): header "# nt ntau size1  sig", then mat, ret, tv and les
 * lines ("ret: i j re im ..."), each number printed like std::ostream with that precision.
 * nt = -1 prints the Matsubara component only. */
int nessi_hm_print_to_file(const char *file, int nt, int ntau, int size1, int sig, const void *ret,
                           const void *les, const void *tv, const void *mat, int precision);

/* The header of a file written by print_to_file: its nt, ntau, size1 and sig. */
int nessi_hm_file_header(const char *file, int *nt, int *ntau, int *size1, int *sig);

/* herm_matrix::read_from_file(file) (cntr_herm_matrix_impl.hpp:1376-1450) into a herm_matrix of
 * the given dimensions: the file's nt must not exceed nt and its ntau and size1 must equal
 * these (libcntr resizes instead; a caller sizes the buffers from nessi_hm_file_header).  Reads
 * mat and time steps 0..nt_file; *sig receives the file's sign. */
int nessi_hm_read_from_file(const char *file, int nt, int ntau, int size1, int *sig, void *ret, void *les,
                            void *tv, void *mat);

/* herm_matrix::read_from_file(nt1, file) (cntr_herm_matrix_impl.hpp:1469-1560): mat and the
 * time steps up to nt1 (ret rows i <= nt1, tv rows i <= nt1, les columns j <= nt1); the rest of
 * the herm_matrix and its sign are left as they are.  nt1 <= nt, nt1 <= nt_file, equal ntau and
 * size1 (the reference's asserts). */
int nessi_hm_read_from_file_nt1(const char *file, int nt1, int nt, int ntau, int size1, void *ret, void *les,
                                void *tv, void *mat);

#ifdef __cplusplus
}
#endif

#endif
