def _upsampled_dft(*args, **kwargs):
    raise NotImplementedError("scikit-image is not available")
