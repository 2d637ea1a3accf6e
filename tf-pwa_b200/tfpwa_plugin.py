"""The engine as an NLL model of the reference package's own registry.

TF-PWA selects the likelihood model of a fit by name
(``tf_pwa/model/model.py:38``, ``register_nll_model``; chosen with
``data: {model: <name>}`` in config.yml and built with the ``nll_model``
section's entries as keyword arguments,
``tf_pwa/config_loader/config_loader.py:587-613``).  :func:`register`
adds a model named ``b200`` whose ``nll_grad_batch`` -- the call
``FCN.nll_grad`` makes (``tf_pwa/model/model.py:1196-1229``) -- runs this
engine: the reference's ``ConfigLoader``, ``get_fcn``, ``fit`` and error
code stay unchanged and only the amplitude/NLL/gradient work moves to the
GPU.

config.yml::

    data:
      model: b200
      ...
    nll_model:
      config_file: config.yml     # this same file (the engine parses it too)
      precision: mixed            # or plain (FP64 throughout)

then ``register()`` once before building the reference's ``ConfigLoader``.
"""
import numpy as np

__all__ = ["register"]


def _momenta(batches, order):
    """(N, n_final, 4) momenta of the reference's data batches (each a dict
    with particle -> {"p": (n, 4)}), finals in ``order``."""
    out = []
    for b in batches:
        parts = {str(k): v for k, v in b["particle"].items()}
        out.append(np.stack([np.asarray(parts[p]["p"], np.float64) for p in order], 1))
    return np.concatenate(out, 0)


def _charges(batches):
    ch = [b.get("charge_conjugation") for b in batches]
    if any(c is None for c in ch):
        return None
    return np.concatenate([np.asarray(c, np.float64) for c in ch])


def register(name="b200"):
    """Register the engine as the reference's NLL model ``name``; returns
    the model class.  Needs the reference package importable."""
    from tf_pwa.model.model import Model, get_nll_model, register_nll_model

    prev = get_nll_model(name, None)
    if prev is not None:
        if getattr(prev, "_b200_engine", False):
            return prev  # registered already (the registry refuses a second entry)
        raise ValueError(f"an NLL model named {name!r} is registered already")

    class B200Model(Model):
        """``nll_grad_batch`` (``tf_pwa/model/model.py:407-449``) through the
        B200 engine.  The first call uploads the events of the batches it
        is given (data with the reference's alpha-scaled weights, MC with
        its normalised weights) and keeps them resident; later calls only
        pass the parameter vector."""

        def __init__(self, amp, w_bkg=1.0, config_file=None, precision="mixed", device=None,
                     **kw):
            super().__init__(amp, w_bkg=w_bkg, **kw)
            if config_file is None:
                raise ValueError("nll_model b200 needs config_file")
            self.config_file = config_file
            self.precision = precision
            self.device = device
            self._fcn = None
            self._cl = None

        def _build(self, data, mcdata, weight, mc_weight):
            from .api import FCN, ConfigLoader

            dev = self.device
            if dev is None:
                import torch

                dev = "cuda" if torch.cuda.is_available() else "cpu"
            cl = ConfigLoader(self.config_file, precision=self.precision)
            order = cl.get_dat_order()
            # under cp_trans the reference's stored momenta of charge -1
            # events are already parity-transformed: only the charge field
            # is needed then
            cp = cl.plan.cp_trans
            w = np.concatenate([np.asarray(x, np.float64) for x in weight])
            wm = np.concatenate([np.asarray(x, np.float64) for x in mc_weight])
            d = cl.data_from_p4(_momenta(data, order), w, device=dev,
                                charge=None if cp else _charges(data))
            m = cl.data_from_p4(_momenta(mcdata, order), wm, device=dev,
                                charge=None if cp else _charges(mcdata))
            if cp:
                ci = cl.plan.charge_index
                for ev, b in ((d, data), (m, mcdata)):
                    c = _charges(b)
                    if ci is not None and c is not None:
                        ev.fields[ci] = c if not hasattr(ev.fields, "device") else \
                            ev.fields.new_tensor(c)
            self._cl = cl
            self._fcn = FCN(cl, d, m, precision=self.precision)
            self._names = list(self.Amp.vm.trainable_vars)
            if self._names != list(cl.vm.trainable_vars):
                raise ValueError("trainable parameters differ between the reference's model "
                                 "and the engine's")

        _b200_engine = True

        def nll_grad_batch(self, data, mcdata, weight, mc_weight):
            data, mcdata = list(data), list(mcdata)
            if self._fcn is None:
                self._build(data, mcdata, list(weight), list(mc_weight))
            vals = {k: float(v) for k, v in self.Amp.vm.get_all_dic().items()}
            self._cl.vm.set_all(vals)
            x = [vals[k] for k in self._names]
            nll, g = self._fcn.nll_grad(x)
            return nll, list(g)

    register_nll_model(name)(B200Model)
    return B200Model
