"""Stand-in for the two scikit-image symbols the reference imports off the path."""
import sys
import types

io = types.ModuleType("skimage.io")
sys.modules["skimage.io"] = io
