"""Data files through the reference-facing loader on the host: the golden
momenta written as the reference's ``E px py pz`` text files (data,
background, phase space), read by ``ConfigLoader.get_data`` (native
multithreaded parser + host kinematics), give the fields that the
reference's own cal_angle produced for the same momenta, and the background
rows get weight -bg_weight (``tf_pwa/config_loader/data.py:149-169,215-232``)."""
import os

import numpy as np
import yaml

from common import CONFIGS, load_golden


def test_config_files_to_reference_fields(tmp_path):
    from tf_pwa_b200.api import ConfigLoader

    g, meta = load_golden("lc2pkpi")
    dic = yaml.safe_load(open(os.path.join(CONFIGS, meta["config"])))
    for kind, key in (("data", "p4_data"), ("bg", "p4_bg"), ("phsp", "p4_mc")):
        f = tmp_path / f"{kind}.dat"
        np.savetxt(f, g[key].reshape(-1, 4), fmt="%.17g")
        dic["data"][kind] = [str(f)]
    dic["data"]["bg_weight"] = meta["extra_data"]["bg_weight"]
    cfg = tmp_path / "config.yml"
    cfg.write_text(yaml.safe_dump(dic))
    cl = ConfigLoader(str(cfg))
    for kind, key in (("data", "fields_data"), ("bg", "fields_bg"), ("phsp", "fields_mc")):
        (d,) = cl.get_data(kind)
        x = d.numpy_fields()
        np.testing.assert_allclose(x, g[key], rtol=0, atol=1e-11)
    (bg,) = cl.get_data("bg")
    assert np.all(np.asarray(bg.weight) == -meta["extra_data"]["bg_weight"])


def test_files_split_by_particle_and_weight_files(tmp_path):
    """A list of files is one sample split by particle (file i holds the
    next particles of dat_order, event by event; ``tf_pwa/data.py:300-365``);
    a list of lists is one sample per inner list; the weight files'
    values are cut to the events read; a ``negtive_idx`` pattern flips the
    sign."""
    from tf_pwa_b200.api import ConfigLoader

    g, meta = load_golden("lc2pkpi")
    p4 = g["p4_data"]
    n = p4.shape[0]
    fa, fb = tmp_path / "p_K.dat", tmp_path / "pi.dat"
    np.savetxt(fa, p4[:, :2].reshape(-1, 4), fmt="%.17g")
    np.savetxt(fb, p4[:, 2:].reshape(-1, 4), fmt="%.17g")
    w = np.linspace(0.5, 1.5, n + 7)  # longer than the sample: cut to n
    wf = tmp_path / "w.dat"
    np.savetxt(wf, w, fmt="%.17g")
    dic = yaml.safe_load(open(os.path.join(CONFIGS, meta["config"])))
    dic["data"] = dict(dic["data"], data=[str(fa), str(fb)], data_weight=str(wf),
                       negtive_idx=["data"])
    cfg = tmp_path / "config.yml"
    cfg.write_text(yaml.safe_dump(dic))
    (d,) = ConfigLoader(str(cfg)).get_data("data")
    np.testing.assert_allclose(d.numpy_fields(), g["fields_data"], rtol=0, atol=1e-11)
    np.testing.assert_array_equal(np.asarray(d.weight), -w[:n])
    # two samples (list of lists), each a single file
    half = n // 2
    f1, f2 = tmp_path / "s1.dat", tmp_path / "s2.dat"
    np.savetxt(f1, p4[:half].reshape(-1, 4), fmt="%.17g")
    np.savetxt(f2, p4[half:].reshape(-1, 4), fmt="%.17g")
    dic["data"] = dict(dic["data"], data=[[str(f1)], [str(f2)]])
    dic["data"].pop("data_weight")
    dic["data"].pop("negtive_idx")
    cfg.write_text(yaml.safe_dump(dic))
    d1, d2 = ConfigLoader(str(cfg)).get_data("data")
    np.testing.assert_allclose(np.concatenate([d1.numpy_fields(), d2.numpy_fields()], 1),
                               g["fields_data"], rtol=0, atol=1e-11)
