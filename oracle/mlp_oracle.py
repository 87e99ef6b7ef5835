"""Test infrastructure: numpy (FP64) restatement of the surrogate network.

The oracle for the device kernels in imate_b200/csrc/slq_mlp.cu
(slq_mlp_forward, slq_mlp_grad, slq_mlp_train): the same 1 -> 64 -> 64 -> 1
tanh network with the same packed parameter layout
W1[64] b1[64] W2[64][64] b2[64] W3[64] b3[1], the mean-squared-error loss and
full-batch Adam.  Only tests/ use it.
"""

import numpy as np

H = 64
P = H + H + H * H + H + H + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + H]; o += H
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


def forward(p, x):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    h1 = np.tanh(np.outer(x, W1) + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h2 @ W3 + b3


def loss_grad(p, x, t):
    """(loss, gradient) of mean_i (net(x_i) - t_i)^2."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    B = x.size
    h1 = np.tanh(np.outer(x, W1) + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    y = h2 @ W3 + b3
    r = y - t
    loss = float(np.mean(r * r))
    dy = 2.0 * r / B
    gW3 = h2.T @ dy
    gb3 = dy.sum()
    dz2 = np.outer(dy, W3) * (1.0 - h2 * h2)
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(axis=0)
    dz1 = (dz2 @ W2) * (1.0 - h1 * h1)
    gW1 = dz1.T @ x
    gb1 = dz1.sum(axis=0)
    g = np.concatenate([gW1, gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, g


def adam(p, x, t, steps, lr, m=None, v=None, steps_done=0, beta1=0.9,
         beta2=0.999, eps=1e-8):
    p = np.array(p, dtype=np.float64)
    m = np.zeros(P) if m is None else np.array(m, dtype=np.float64)
    v = np.zeros(P) if v is None else np.array(v, dtype=np.float64)
    losses = []
    for k in range(steps):
        loss, g = loss_grad(p, x, t)
        losses.append(loss)
        m = beta1 * m + (1 - beta1) * g
        v = beta2 * v + (1 - beta2) * g * g
        s = steps_done + k + 1
        mh = m / (1 - beta1 ** s)
        vh = v / (1 - beta2 ** s)
        p = p - lr * mh / (np.sqrt(vh) + eps)
    return p, m, v, np.asarray(losses)
