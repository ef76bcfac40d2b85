"""CPU (numpy, FP64 arithmetic) restatement of the surrogate MLP's forward and
backward passes with the BF16 roundings of the GPU path at the same points
(operands of every GEMM), used to check the GPU gradients.  Test
infrastructure only."""
import numpy as np

C = 0.7978845608028654


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    a = np.asarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1 + np.tanh(C * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(C * (x + 0.044715 * x ** 3))
    return 0.5 * (1 + t) + 0.5 * x * (1 - t * t) * C * (1 + 3 * 0.044715 * x * x)


def forward_backward(X, W, b, T, w):
    """X [B, 160] (BF16 values), W = [W1, W2, W3] (FP32 masters), b biases,
    T [B, 80] targets, w [80] loss weights.  Returns loss, Y, dW, db with the
    GPU's BF16 rounding of GEMM operands."""
    Wb = [bf16(m) for m in W]
    B = X.shape[0]
    Z1 = X @ Wb[0].T + b[0]
    H1 = bf16(gelu(Z1))
    Z2 = H1 @ Wb[1].T + b[1]
    H2 = bf16(gelu(Z2))
    Y = H2 @ Wb[2].T + b[2]
    e = Y - T
    loss = float((w * e * e).sum())
    dY32 = (2.0 / B) * w * e
    dY = bf16(dY32)
    dW3 = dY.T @ H2
    db3 = dY32.sum(0)
    dZ2 = (dY @ Wb[2]) * gelu_grad(Z2)
    dZ2b = bf16(dZ2)
    dW2 = dZ2b.T @ H1
    db2 = dZ2.sum(0)
    dZ1 = (dZ2b @ Wb[1]) * gelu_grad(Z1)
    dW1 = bf16(dZ1).T @ X
    db1 = dZ1.sum(0)
    return loss, Y, [dW1, dW2, dW3], [db1, db2, db3]
