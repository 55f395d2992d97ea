"""Host-side contour functions with libcntr's memory layout.

``herm_matrix`` mirrors ``cntr::herm_matrix<double>``
(libcntr/cntr/cntr_herm_matrix_decl.hpp:44-301): the retarded and lesser
components are packed triangles, tv is a (nt+1) x (ntau+1) rectangle and mat a
vector, each element a row-major size1 x size1 block of complex<double>
(offsets cntr_herm_matrix_impl.hpp:457-477):

    ret(t,t'), t' <= t : (t(t+1)/2 + t')
    les(t,t'), t <= t' : (t'(t'+1)/2 + t)
    tv(t,tau)          : t(ntau+1) + tau
    mat(tau)           : tau

``function`` mirrors ``cntr::function<double>`` (cntr_function_decl.hpp:45):
(nt+2) blocks with ``ptr(t) = data + (t+1) s^2`` so that t = -1 is the
Matsubara value.

The arrays are contiguous numpy ``complex128`` arrays, so their base pointers
are exactly what ``retptr(0,0)``, ``lesptr(0,0)``, ``tvptr(0,0)`` and
``matptr(0)`` return in libcntr; the C ABI of ``libnessi_gpu.so`` takes them as
plain pointers.
"""
import numpy as np

CPLX = np.complex128


def _tri(nt):
    return (nt + 1) * (nt + 2) // 2


class herm_matrix:
    """Two-time contour function G(t,t') with hermitian symmetry (libcntr herm_matrix)."""

    def __init__(self, nt=-1, ntau=0, size1=1, sig=-1):
        if size1 < 1 or nt < -1 or ntau < 0 or sig not in (-1, 1):
            raise ValueError("herm_matrix: bad dimensions nt=%d ntau=%d size1=%d sig=%d"
                             % (nt, ntau, size1, sig))
        self.nt, self.ntau, self.size1, self.sig = nt, ntau, size1, sig
        s = size1
        self.mat = np.zeros((ntau + 1, s, s), CPLX)
        if nt >= 0:
            self.ret = np.zeros((_tri(nt), s, s), CPLX)
            self.les = np.zeros((_tri(nt), s, s), CPLX)
            self.tv = np.zeros((nt + 1, ntau + 1, s, s), CPLX)
        else:
            self.ret = np.zeros((0, s, s), CPLX)
            self.les = np.zeros((0, s, s), CPLX)
            self.tv = np.zeros((0, ntau + 1, s, s), CPLX)

    # --- sizes ---------------------------------------------------------------------
    @property
    def size(self):
        return self.size1

    def element_size(self):
        return self.size1 * self.size1

    # --- offsets (element units) ---------------------------------------------------
    @staticmethod
    def ret_index(t, t1):
        return t * (t + 1) // 2 + t1

    @staticmethod
    def les_index(t, t1):
        return t1 * (t1 + 1) // 2 + t

    # --- element access ------------------------------------------------------------
    def get_ret(self, t, t1):
        """G^R(t,t') for any t,t' using the hermitian continuation for t < t'."""
        if t1 <= t:
            return self.ret[self.ret_index(t, t1)].copy()
        return -self.ret[self.ret_index(t1, t)].conj().T

    def get_les(self, t, t1):
        if t <= t1:
            return self.les[self.les_index(t, t1)].copy()
        return -self.les[self.les_index(t1, t)].conj().T

    def get_tv(self, t, tau):
        return self.tv[t, tau].copy()

    def get_mat(self, tau):
        return self.mat[tau].copy()

    def ret_row(self, t):
        """View of ret(t, 0..t) (contiguous, libcntr retptr(t,0))."""
        i0 = self.ret_index(t, 0)
        return self.ret[i0:i0 + t + 1]

    def les_col(self, t1):
        """View of les(0..t1, t1) (contiguous, libcntr lesptr(0,t1))."""
        i0 = self.les_index(0, t1)
        return self.les[i0:i0 + t1 + 1]

    # --- time-step operations (cntr_herm_matrix_impl.hpp:2098-2725) ----------------
    def smul(self, tstp, w):
        if tstp == -1:
            self.mat *= w
        else:
            self.ret_row(tstp)[...] *= w
            self.tv[tstp] *= w
            self.les_col(tstp)[...] *= w

    def set_timestep(self, tstp, other):
        if tstp == -1:
            self.mat[...] = other.mat
        else:
            self.ret_row(tstp)[...] = other.ret_row(tstp)
            self.tv[tstp] = other.tv[tstp]
            self.les_col(tstp)[...] = other.les_col(tstp)

    def incr_timestep(self, tstp, other, alpha=1.0):
        if tstp == -1:
            self.mat += alpha * other.mat
        else:
            self.ret_row(tstp)[...] += alpha * other.ret_row(tstp)
            self.tv[tstp] += alpha * other.tv[tstp]
            self.les_col(tstp)[...] += alpha * other.les_col(tstp)

    def left_multiply(self, tstp, f, weight=1.0):
        """C(t,t') -> weight f(t) C(t,t') at time step tstp (cntr_herm_matrix_impl.hpp:2955-2995):
        f(-1) on mat, f(tstp) on ret(tstp, .) and tv(tstp, .), f(m) on les(m, tstp).  ``f`` is a
        cntr::function or its (nt+2, s, s) data, t = -1 first."""
        F = f.data if isinstance(f, function) else np.asarray(f)
        if tstp == -1:
            self.mat[...] = weight * np.einsum("ab,mbc->mac", F[0], self.mat)
            return
        self.ret_row(tstp)[...] = weight * np.einsum("ab,mbc->mac", F[tstp + 1], self.ret_row(tstp))
        self.tv[tstp] = weight * np.einsum("ab,mbc->mac", F[tstp + 1], self.tv[tstp])
        self.les_col(tstp)[...] = weight * np.einsum("mab,mbc->mac", F[1:tstp + 2], self.les_col(tstp))

    def right_multiply(self, tstp, f, weight=1.0):
        """C(t,t') -> weight C(t,t') f(t') at time step tstp (cntr_herm_matrix_impl.hpp:3206-3246):
        f(-1) on mat and tv(tstp, .), f(m) on ret(tstp, m), f(tstp) on les(m, tstp)."""
        F = f.data if isinstance(f, function) else np.asarray(f)
        if tstp == -1:
            self.mat[...] = weight * np.einsum("mab,bc->mac", self.mat, F[0])
            return
        self.ret_row(tstp)[...] = weight * np.einsum("mab,mbc->mac", self.ret_row(tstp), F[1:tstp + 2])
        self.tv[tstp] = weight * np.einsum("mab,bc->mac", self.tv[tstp], F[0])
        self.les_col(tstp)[...] = weight * np.einsum("mab,bc->mac", self.les_col(tstp), F[tstp + 1])

    def set_matrixelement(self, tstp, i1, i2, other, j1=0, j2=0):
        """self(i1,i2) <- other(j1,j2) at one time step (cntr_herm_matrix_impl.hpp set_matrixelement)."""
        if tstp == -1:
            self.mat[:, i1, i2] = other.mat[:, j1, j2]
        else:
            self.ret_row(tstp)[:, i1, i2] = other.ret_row(tstp)[:, j1, j2]
            self.tv[tstp, :, i1, i2] = other.tv[tstp, :, j1, j2]
            self.les_col(tstp)[:, i1, i2] = other.les_col(tstp)[:, j1, j2]

    def get_timestep(self, tstp):
        """Packed slice [ret(n,0..n) | tv(n,0..ntau) | les(0..n,n)]
        (cntr_herm_matrix_timestep_decl.hpp:67-75); mat for tstp == -1."""
        if tstp == -1:
            return self.mat.copy()
        return np.concatenate([self.ret_row(tstp), self.tv[tstp], self.les_col(tstp)])

    def set_timestep_data(self, tstp, data):
        if tstp == -1:
            self.mat[...] = data
            return
        n1 = tstp + 1
        self.ret_row(tstp)[...] = data[:n1]
        self.tv[tstp] = data[n1:n1 + self.ntau + 1]
        self.les_col(tstp)[...] = data[n1 + self.ntau + 1:]

    def copy(self):
        c = herm_matrix(self.nt, self.ntau, self.size1, self.sig)
        c.ret[...] = self.ret
        c.les[...] = self.les
        c.tv[...] = self.tv
        c.mat[...] = self.mat
        return c



class function:
    """Time-local matrix function f(t), t = -1..nt (libcntr cntr::function)."""

    def __init__(self, nt=-1, size1=1):
        self.nt, self.size1 = nt, size1
        self.data = np.zeros((nt + 2, size1, size1), CPLX)

    def ptr(self, t):
        return self.data[t + 1]

    def set_value(self, t, M):
        self.data[t + 1] = M

    def set_constant(self, M):
        self.data[...] = M

    def get_value(self, t):
        return self.data[t + 1].copy()


def distance_norm2(tstp, g1, g2):
    """Sum of Frobenius norms of element differences at one time step
    (cntr_utilities_impl.hpp:607-650)."""
    if tstp == -1:
        return float(np.sum(np.sqrt(np.sum(np.abs(g1.mat - g2.mat) ** 2, axis=(1, 2)))))
    d = 0.0
    for a, b in ((g1.ret_row(tstp), g2.ret_row(tstp)), (g1.tv[tstp], g2.tv[tstp]),
                 (g1.les_col(tstp), g2.les_col(tstp))):
        d += float(np.sum(np.sqrt(np.sum(np.abs(a - b) ** 2, axis=(1, 2)))))
    return d
