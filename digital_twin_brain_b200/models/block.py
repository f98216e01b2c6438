"""Drop-in replacement of the reference's ``models/block.py`` ``block`` class.

``block(node_property, w_uij, delta_t, src)`` builds the network on the GPU
(libdtb) and ``run(noise_rate, isolated)`` advances it one time step with
the CUDA kernels, returning the per-subblock spike sums and mean membrane
potentials exactly like ``models/block.py:116-150``.  The public state
tensors ``V_i``, ``J_ui``, ``I_ui``, ``I_syn``, ``t_ik_last``, ``active`` and
``t`` are read back from the device on access.

Differences from the reference, by design:

* Background noise comes from the counter-based Philox4x32-10 stream keyed by
  ``seed`` (step index = counter), not from torch's global CPU generator.
  With torch.rand replaced by the same stream, results are bit-identical in
  ``mode="pull"`` (the default): the pull kernel accumulates every row in the
  order torch.sparse.mm does.  ``mode="push"`` / ``"auto"`` use float atomics
  and agree to float32 rounding.
* A dense ``w_uij`` is accepted and converted to its nonzero entries; dense
  ``torch.matmul`` summation order is not reproduced (rounding-level match).
* ``src`` (input neurons replaying a spike raster, models/block.py:37-50,
  104-109) is held on the device; as in the reference, the input neurons are
  those without incoming synapses, a raster of T columns serves T - 1 steps
  and the step after that raises IndexError.
"""
from __future__ import annotations

import numpy as np
import torch

from .._lib import (FIELD_ACTIVE, FIELD_I_SYN, FIELD_I_UI, FIELD_J, FIELD_NEW_ACTIVE, FIELD_T, FIELD_T_LAST,
                    FIELD_V)
from ..network import Network


def coo_entries(w_uij: torch.Tensor):
    """[4,N,N] weights -> synapse entries (post, pre, kind, weight[S,2]) in torch.sparse.mm order.

    generation/read_block.py:68-74 stores every synapse as two consecutive COO
    entries (channel c and c+1, c in {0,2}); those pairs become one synapse.
    Any other entry becomes a synapse that adds its value to its own channel
    and +0 to the partner channel, which leaves every channel's sum and its
    order unchanged.
    """
    if w_uij.is_sparse:
        idx = w_uij._indices().cpu().numpy()
        val = w_uij._values().detach().cpu().float().numpy()
    else:
        W = w_uij.detach().cpu().float()
        nz = torch.nonzero(W)
        # order by (post, pre, channel): dense rows have no nnz order of their own
        order = np.lexsort((nz[:, 0].numpy(), nz[:, 2].numpy(), nz[:, 1].numpy()))
        nz = nz[torch.from_numpy(order)]
        idx = nz.T.numpy()
        val = W[nz[:, 0], nz[:, 1], nz[:, 2]].numpy()
    c, post, pre = idx[0].astype(np.int64), idx[1].astype(np.int64), idx[2].astype(np.int64)
    n = c.size
    if n and n % 2 == 0:
        ce, co = c[0::2], c[1::2]
        if (((ce == 0) | (ce == 2)) & (co == ce + 1) & (post[0::2] == post[1::2]) & (pre[0::2] == pre[1::2])).all():
            w = np.stack([val[0::2], val[1::2]], axis=1).astype(np.float32)
            return post[0::2], pre[0::2], ce.astype(np.uint8), w
    if n and (c.min() < 0 or c.max() > 3):
        raise ValueError("w_uij channel index must be in 0..3")
    w = np.zeros((n, 2), np.float32)
    w[np.arange(n), c & 1] = val
    return post, pre, (c & 2).astype(np.uint8), w


def decay_of(node_property: torch.Tensor, delta_t: float) -> np.ndarray:
    """exp(-dt/tau_ui) evaluated as models/block.py:71 does, returned as [N,4]."""
    tau = node_property.detach().cpu().float().transpose(0, 1)[18:22]
    d = torch.exp(-delta_t / tau)
    return np.ascontiguousarray(d.transpose(0, 1).numpy(), np.float32)


class block:
    """GPU-backed ``block`` (models/block.py:5-177).

    Extra keyword arguments: ``seed`` (Philox noise key), ``device`` (CUDA
    ordinal, default the current device), ``mode`` ("pull" bit-exact default,
    "push", "auto"), ``build_push`` (also build the presynaptic CSR).
    """

    def __init__(self, node_property, w_uij, delta_t=1, src=None, *, seed: int = 0, device: int | None = None,
                 mode: str = "pull", build_push: bool = True):
        assert len(w_uij.shape) == 3
        N = w_uij.shape[1]
        K = w_uij.shape[0]
        assert K == 4, "w_uij must have 4 channels (AMPA, NMDA, GABAa, GABAb)"
        assert node_property.shape[0] == N and node_property.shape[1] == 22
        self.src = src
        self.src_neuron = None
        self.iter = None
        self.delta_t = delta_t
        self.mode = mode
        self._out_device = w_uij.device
        if device is None:
            device = torch.cuda.current_device()
        post, pre, kind, w = coo_entries(w_uij)
        prop = node_property.detach().cpu().float().numpy()
        self._net = Network.from_arrays(prop, post, pre, kind, w, dt=float(delta_t), seed=seed,
                                        decay=decay_of(node_property, delta_t), device=device,
                                        build_push=build_push)
        if src is not None:
            # neurons without any incoming entry (models/block.py:41-47)
            idx = np.setdiff1d(np.arange(N, dtype=np.int64), np.unique(post))
            self.src_neuron = torch.from_numpy(idx)
            assert self.src_neuron.shape[0] == src.shape[0]
            self.iter = 0
            self._net.set_input_spikes(idx, torch.as_tensor(src).cpu().numpy().astype(np.uint8))
        self._set_property_views(node_property)

    def _set_property_views(self, node_property):
        p = node_property.detach().float()
        (E_I, blocked_in_stat, I_extern_Input, sub_idx, C, T_ref, g_Li, V_L, V_th, V_reset, g_ui, V_ui,
         tau_ui) = p.transpose(0, 1).split([1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 4, 4, 4])
        self.I_extern_Input = I_extern_Input.squeeze(0)
        self.V_ui, self.tau_ui, self.g_ui = V_ui, tau_ui, g_ui
        self.g_Li, self.V_L, self.C = g_Li.squeeze(0), V_L.squeeze(0), C.squeeze(0)
        self.sub_idx = sub_idx.squeeze(0)
        self.V_th, self.V_reset, self.T_ref = V_th.squeeze(0), V_reset.squeeze(0), T_ref.squeeze(0)

    @property
    def network(self) -> Network:
        return self._net

    def _out(self, a: np.ndarray) -> torch.Tensor:
        return torch.from_numpy(a).to(self._out_device)

    # ---------------------------------------------------------------- step
    def _take_src(self, n: int):
        if self.src is None:
            return
        if self.iter + n >= self.src.shape[1]:
            # models/block.py:107 reads src[:, iter + 1] after replaying column iter
            raise IndexError(f"index {self.src.shape[1]} is out of bounds for dimension 1 with size "
                             f"{self.src.shape[1]}")
        self.iter += n

    def run(self, noise_rate=0.01, isolated=False):
        """One time step (models/block.py:116-150): (spike sum, mean V) per subblock."""
        self._take_src(1)
        s, m, _ = self._net.run(1, noise_rate=noise_rate, isolated=isolated, mode=self.mode, out="host")
        return self._out(s[0]), self._out(m[0])

    def run_steps(self, n_steps: int, noise_rate=0.01, isolated=False):
        """n_steps calls of run() in one native call; per-step results stacked."""
        self._take_src(n_steps)
        s, m, _ = self._net.run(n_steps, noise_rate=noise_rate, isolated=isolated, mode=self.mode, out="host")
        return self._out(s), self._out(m)

    # ---------------------------------------------------------------- state
    @property
    def V_i(self) -> torch.Tensor:
        return self._out(self._net.get(FIELD_V))

    @property
    def J_ui(self) -> torch.Tensor:
        return self._out(self._net.get(FIELD_J))

    @property
    def I_ui(self) -> torch.Tensor:
        return self._out(self._net.get(FIELD_I_UI))

    @property
    def I_syn(self) -> torch.Tensor:
        return self._out(self._net.get(FIELD_I_SYN))

    @property
    def t_ik_last(self) -> torch.Tensor:
        return self._out(self._net.get(FIELD_T_LAST))

    @property
    def active(self) -> torch.Tensor:
        return self._out(self._net.get(FIELD_ACTIVE).astype(bool))

    @property
    def new_active(self) -> torch.Tensor:
        return self._out(self._net.get(FIELD_NEW_ACTIVE).astype(bool))

    @property
    def t(self) -> torch.Tensor:
        return torch.tensor(self._net.get(FIELD_T), dtype=torch.float32, device=self._out_device)

    # ---------------------------------------------------------------- updates
    def update_property(self, node_property):
        """models/block.py:152-170."""
        prop = node_property.detach().cpu().float().numpy()
        self._net.update_property(prop, decay_of(node_property, self.delta_t))
        self._set_property_views(node_property)
        return True

    def update_conn_weight(self, conn_idx, conn_weight):
        """models/block.py:172-177: conn_idx [3, X] (channel, post, pre), conn_weight [X]."""
        idx = torch.as_tensor(conn_idx).cpu().numpy()
        val = torch.as_tensor(conn_weight).detach().cpu().float().numpy().reshape(-1)
        if idx.shape[0] == 4:
            idx = idx[:3]
        self._net.update_conn_weight(idx[0], idx[1], idx[2], val)
        return True
