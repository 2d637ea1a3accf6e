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


def test_weight_files_follow_the_event_files(tmp_path):
    """Two data files and one weight file: each file's events take the next
    slice of the weights; a ``negtive_idx`` pattern flips the sign."""
    from tf_pwa_b200.api import ConfigLoader

    g, meta = load_golden("lc2pkpi")
    p4 = g["p4_data"]
    half = p4.shape[0] // 2
    files = []
    for i, part in enumerate((p4[:half], p4[half:])):
        f = tmp_path / f"data{i}.dat"
        np.savetxt(f, part.reshape(-1, 4), fmt="%.17g")
        files.append(str(f))
    w = np.linspace(0.5, 1.5, p4.shape[0])
    wf = tmp_path / "w.dat"
    np.savetxt(wf, w, fmt="%.17g")
    dic = yaml.safe_load(open(os.path.join(CONFIGS, meta["config"])))
    dic["data"] = {"data": files, "data_weight": str(wf), "negtive_idx": ["data"]}
    cfg = tmp_path / "config.yml"
    cfg.write_text(yaml.safe_dump(dic))
    d0, d1 = ConfigLoader(str(cfg)).get_data("data")
    np.testing.assert_array_equal(np.asarray(d0.weight), -w[:half])
    np.testing.assert_array_equal(np.asarray(d1.weight), -w[half:])
