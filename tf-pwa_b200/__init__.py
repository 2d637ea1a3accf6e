"""B200-native engine for TF-PWA's unbinned amplitude-fit hot path.

Import name ``tf_pwa_b200`` (the source directory is ``tf-pwa_b200``)."""
__version__ = "0.1.0"
