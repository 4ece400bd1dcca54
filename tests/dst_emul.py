"""numpy restatement of the tensor-core DST preconditioner's arithmetic (test
helper): every transform pass rounds its input to BF16 (via FP32, round to
nearest even), multiplies by the BF16-rounded DST-I matrix with wide
accumulation, and the scaled pass divides by the separable eigenvalues."""
import numpy as np


def bf16(x):
    """Round to BF16 (through FP32, round to nearest even); returns float64."""
    u = np.asarray(x, np.float64).astype(np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def dst_matrix(n):
    j = np.arange(1, n + 1)
    return np.sqrt(2.0 / (n + 1)) * np.sin(np.pi * np.outer(j, j) / (n + 1))


def eigvals(n, c):
    j = np.arange(1, n + 1)
    return c * 4.0 * np.sin(np.pi * j / (2.0 * (n + 1))) ** 2


def apply_exact(R, nx, ny, cx, cy, shift):
    """T R in FP64 for R of shape (nx*ny, B), lattice row-major (iy, ix)."""
    B = R.shape[1]
    G = R.reshape(ny, nx, B)
    Sx, Sy = dst_matrix(nx), dst_matrix(ny)
    lam = eigvals(ny, cy)[:, None] + eigvals(nx, cx)[None, :] + shift
    H = np.einsum("ij,yjb->yib", Sx, G)
    H = np.einsum("ij,jxb->ixb", Sy, H) / lam[:, :, None]
    H = np.einsum("ij,jxb->ixb", Sy, H)
    H = np.einsum("ij,yjb->yib", Sx, H)
    return H.reshape(nx * ny, B)


def apply_bf16(R, nx, ny, cx, cy, shift):
    """T R with the kernel's roundings (BF16 operands, wide accumulation)."""
    B = R.shape[1]
    G = R.reshape(ny, nx, B)
    Sx, Sy = bf16(dst_matrix(nx)), bf16(dst_matrix(ny))
    lam = (eigvals(ny, cy)[:, None] + (eigvals(nx, cx) + shift)[None, :])
    H = bf16(np.einsum("ij,yjb->yib", Sx, bf16(G)))
    H = bf16(np.einsum("ij,jxb->ixb", Sy, H) / lam[:, :, None])
    H = bf16(np.einsum("ij,jxb->ixb", Sy, H))
    H = np.einsum("ij,yjb->yib", Sx, H)
    return H.reshape(nx * ny, B)
