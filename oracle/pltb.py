"""The reference's .pltb file format, restated for tests.

Matrix4D::writeToBinaryFile / readFromBinaryFile (src/Matrix.cpp:5700-5720,
5780-5808): four native int32 sizes (w, x, y, z), then w*x*y*z values in the
Matrix4D plane-array order ([w][x][y][z], z fastest), native byte order."""
import numpy as np


def write(path, arr):
    a = np.ascontiguousarray(arr, dtype=np.float64)
    with open(path, "wb") as f:
        f.write(np.asarray(a.shape, dtype=np.int32).tobytes())
        f.write(a.tobytes())


def read(path):
    with open(path, "rb") as f:
        shape = tuple(np.frombuffer(f.read(16), dtype=np.int32))
        data = np.frombuffer(f.read(), dtype=np.float64)
    return data.reshape(shape)
