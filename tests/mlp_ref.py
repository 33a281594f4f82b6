"""numpy restatement of the controller MLP (tanh hidden layers, linear
output, mean squared error) for checking the device kernels: forward and
analytic gradient in f64, parameters in the device order W1, b1, W2, b2, W3, b3."""
import numpy as np


def unpack(p, n_in, h, n_out):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + h * n_in].reshape(h, n_in); o += h * n_in
    b1 = p[o:o + h]; o += h
    W2 = p[o:o + h * h].reshape(h, h); o += h * h
    b2 = p[o:o + h]; o += h
    W3 = p[o:o + n_out * h].reshape(n_out, h); o += n_out * h
    b3 = p[o:o + n_out]
    return W1, b1, W2, b2, W3, b3


def forward(p, x, n_in, h, n_out):
    W1, b1, W2, b2, W3, b3 = unpack(p, n_in, h, n_out)
    x = np.asarray(x, dtype=np.float64)
    a1 = np.tanh(x @ W1.T + b1)
    a2 = np.tanh(a1 @ W2.T + b2)
    return a2 @ W3.T + b3, (x, a1, a2)


def loss_and_grad(p, x, t, n_in, h, n_out):
    W1, b1, W2, b2, W3, b3 = unpack(p, n_in, h, n_out)
    y, (x, a1, a2) = forward(p, x, n_in, h, n_out)
    B = x.shape[0]
    r = y - np.asarray(t, dtype=np.float64)
    loss = float(np.sum(r * r) / B)
    d3 = 2.0 * r / B
    gW3 = d3.T @ a2
    gb3 = d3.sum(axis=0)
    d2 = (d3 @ W3) * (1.0 - a2 * a2)
    gW2 = d2.T @ a1
    gb2 = d2.sum(axis=0)
    d1 = (d2 @ W2) * (1.0 - a1 * a1)
    gW1 = d1.T @ x
    gb1 = d1.sum(axis=0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
