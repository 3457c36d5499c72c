"""Host-side file helpers of the visual centre searches.

Restate, for the two ``find_center_visual_*`` functions, the behaviour of
``algotom/io/loadersaver.py`` that they rely on: ``make_folder_name``
(``:297-326``: the next unused ``<prefix>_<number>`` folder name, counting
the existing ``<prefix>_*`` entries) and ``save_image`` (``:382-418``: a 2-D
array written by Pillow, float data as a 32-bit float TIFF, parent folders
created).  Plain host I/O around the device reconstructions.
"""
from pathlib import Path

import numpy as np


def make_folder_name(folder_path, name_prefix="Output", zero_prefix=5):
    folder_path = Path(folder_path)
    scan_name_prefix = name_prefix + "_"
    num_folder_new = len(list(folder_path.glob(f"{scan_name_prefix}*"))) + 1
    scan_name = scan_name_prefix + f"{num_folder_new:0{zero_prefix}}"
    while (folder_path / scan_name).is_dir():
        num_folder_new += 1
        scan_name = scan_name_prefix + f"{num_folder_new:0{zero_prefix}}"
    return scan_name


def save_image(file_path, mat):
    """Write a 2-D real array as a TIFF (``.tif`` / ``.tiff``) or, for other
    extensions, as 8-bit levels of its range, creating the folder."""
    from PIL import Image
    file_path = Path(file_path).resolve()
    mat = np.asarray(mat)
    if file_path.suffix not in (".tif", ".tiff"):
        mat = np.uint8(255.0 * (mat - np.min(mat)) /
                       (np.max(mat) - np.min(mat)))
    elif "complex" in str(mat.dtype):
        raise ValueError(f"Can't save to tiff with format: {mat.dtype}")
    folder = file_path.parent if file_path.suffix else file_path
    try:
        folder.mkdir(parents=True, exist_ok=True)
    except Exception as e:
        raise ValueError(f"Can't create : {folder}. Error: {e}")
    try:
        Image.fromarray(mat).save(file_path)
    except Exception as error:
        raise ValueError(f"Couldn't write to file: {file_path}. "
                         f"Error {error}")
    return file_path
