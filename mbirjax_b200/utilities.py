"""Synthetic phantoms and sinograms for the benchmark workloads.

The workloads are seeded synthetic stand-ins (there is no public dataset behind the benchmark): volumes of
axis-aligned ellipsoids with centres uniform in the inner 70% of the volume, semi-axes uniform in [5, 40]
voxels and densities uniform in [0.1, 1], summed where they overlap (the same construction as the
reference's ``add_ellipsoid``, ``utilities.py:856-895``, without rotation).  Generation runs with torch on
whatever device the caller names (the CPU in tests, the GPU for the large configurations).

Also here: the reference's test phantoms (the low-dynamic-range 3D Shepp-Logan of
``gen_modified_3d_sl_phantom`` and the sheared cube of ``gen_cube_phantom``), the translation-vector raster of
its translation experiments and its HDF5 helpers ``save_data_hdf5`` / ``load_data_hdf5`` (which need h5py).
"""
import math
import os

import numpy as np
import torch


def gen_ellipsoid_phantom(recon_shape, num_ellipsoids, seed, device='cpu', dtype=torch.float32):
    rng = np.random.default_rng(seed)
    nr, nc, ns = recon_shape
    shape = np.array([nr, nc, ns], dtype=np.float64)
    centres = rng.uniform(0.15, 0.85, size=(num_ellipsoids, 3)) * (shape - 1)
    axes = rng.uniform(5.0, 40.0, size=(num_ellipsoids, 3))
    dens = rng.uniform(0.1, 1.0, size=num_ellipsoids)
    out = torch.zeros((nr, nc, ns), dtype=dtype, device=device)
    i = torch.arange(nr, device=device, dtype=torch.float64)[:, None, None]
    j = torch.arange(nc, device=device, dtype=torch.float64)[None, :, None]
    k = torch.arange(ns, device=device, dtype=torch.float64)[None, None, :]
    for c, a, d in zip(centres, axes, dens):
        # bounding box to keep large volumes cheap
        lo = np.maximum(np.floor(c - a), 0).astype(int)
        hi = np.minimum(np.ceil(c + a) + 1, shape).astype(int)
        if np.any(hi <= lo):
            continue
        ii, jj, kk = i[lo[0]:hi[0]], j[:, lo[1]:hi[1]], k[:, :, lo[2]:hi[2]]
        inside = ((ii - c[0]) / a[0]) ** 2 + ((jj - c[1]) / a[1]) ** 2 + ((kk - c[2]) / a[2]) ** 2 <= 1.0
        out[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] += float(d) * inside.to(dtype)
    return out


# (x0, y0, z0, a, b, c, angle in degrees, intensity) of the ellipsoids of the low-dynamic-range Shepp-Logan
# phantom, in the order they are added (utilities.py:684-694 of the reference).  x runs along recon rows, y along
# columns and z along slices, each over [-1, 1].
_SHEPP_LOGAN_LOW_DYNAMIC_RANGE = (
    (0.0, 0.0, 0.0, 0.69, 0.92, 0.9, 0.0, 1.0),
    (0.0, 0.0184, 0.0, 0.6624, 0.874, 0.88, 0.0, -0.8),
    (0.22, 0.0, 0.0, 0.41, 0.16, 0.21, 108.0, -0.2),
    (-0.22, 0.0, 0.0, 0.31, 0.11, 0.22, 72.0, -0.2),
    (0.0, 0.35, 0.0, 0.21, 0.25, 0.5, 0.0, 0.1),
    (0.0, 0.1, 0.0, 0.046, 0.046, 0.046, 0.0, 0.1),
    (0.0, -0.1, 0.0, 0.046, 0.046, 0.046, 0.0, 0.1),
    (-0.08, -0.605, 0.0, 0.046, 0.023, 0.02, 0.0, 0.1),
    (0.0, -0.605, 0.0, 0.023, 0.023, 0.02, 0.0, 0.1),
)


def generate_3d_shepp_logan_low_dynamic_range(phantom_shape, device='cpu'):
    """The reference's low-dynamic-range 3D Shepp-Logan phantom (utilities.py:658-696): float32 (rows, cols,
    slices), each ellipsoid adding its intensity where (xr/a)^2 + (yr/b)^2 + ((z-z0)/c)^2 <= 1, with (xr, yr) the
    in-plane offset rotated by the ellipsoid's angle.  The slices are filled in blocks, so the peak extra memory
    is about 64 M elements whatever the volume."""
    nr, nc, ns = (int(v) for v in phantom_shape)
    f32 = torch.float32
    x = torch.linspace(-1, 1, nr, dtype=f32, device=device)[:, None]
    y = torch.linspace(-1, 1, nc, dtype=f32, device=device)[None, :]
    z = torch.linspace(-1, 1, ns, dtype=f32, device=device)
    phantom = torch.zeros((nr, nc, ns), dtype=f32, device=device)
    block = max(1, (1 << 26) // max(1, nr * nc))
    for x0, y0, z0, a, b, c, angle, intensity in _SHEPP_LOGAN_LOW_DYNAMIC_RANGE:
        t = torch.tensor(math.radians(angle), dtype=f32)
        cos_t, sin_t = float(torch.cos(t)), float(torch.sin(t))
        xr = cos_t * (x - x0) + sin_t * (y - y0)
        yr = -sin_t * (x - x0) + cos_t * (y - y0)
        xy_norm = (xr ** 2 / a ** 2 + yr ** 2 / b ** 2)[:, :, None]
        z_norm = (z - z0) ** 2 / c ** 2
        for k0 in range(0, ns, block):
            k1 = min(ns, k0 + block)
            phantom[:, :, k0:k1] += intensity * ((xy_norm + z_norm[k0:k1]) <= 1).to(f32)
    return phantom


def gen_cube_phantom(recon_shape, device='cpu'):
    """The reference's cube phantom (utilities.py:1034-1056): a block of a quarter of the rows and columns,
    centred, with value 1 / max(its rows, its cols), whose columns shift right by int(slice * cols / num_slices)
    from slice to slice."""
    nr, nc, ns = (int(v) for v in recon_shape[:3])
    rows, cols = nr // 4, nc // 4
    phantom = np.zeros((nr, nc, ns))
    r0, r1 = (nr - rows) // 2, (nr + rows) // 2
    c0, c1 = (nc - cols) // 2, (nc + cols) // 2
    for k in range(ns):
        shift = int(k * cols / ns)
        phantom[r0:r1, shift + c0:shift + c1, k] = 1.0 / max(rows, cols)
    return torch.as_tensor(phantom, dtype=torch.float32, device=device)


def gen_translation_phantom(recon_shape, option, words, fill_rate=0.05, font_size=20):
    """The reference's translation-tomography phantoms (utilities.py:696-717): 'dots' (gen_dot_phantom) or
    'text' (gen_text_phantom); float32 NumPy (rows, cols, slices)."""
    if option == 'dots':
        return gen_dot_phantom(recon_shape, fill_rate)
    if option == 'text':
        return gen_text_phantom(recon_shape, words, font_size)
    raise ValueError(f"Unsupported phantom option: {option}")


def gen_dot_phantom(recon_shape, fill_rate):
    """utilities.py:720-747: the middle two thirds of the recon rows (a sixth of the rows left empty at each end)
    each get int(cols * slices * fill_rate) ones at distinct random (col, slice) positions.  Like the reference it
    seeds np.random with 42 and draws with np.random.choice, so the volume (and the global np.random state after
    it) is the reference's."""
    np.random.seed(42)
    phantom = np.zeros(recon_shape, dtype=np.float32)
    pad = recon_shape[0] // 6
    row_size = recon_shape[1] * recon_shape[2]
    ones_per_row = int(row_size * fill_rate)
    for r in range(pad, recon_shape[0] - pad):
        flat = phantom[r].reshape(-1)
        flat[np.random.choice(row_size, ones_per_row, replace=False)] = 1.0
    return phantom


_FALLBACK_FONTS = ("/System/Library/Fonts/Supplemental/Arial.ttf", "/Library/Fonts/Arial.ttf",
                   "/usr/share/fonts/truetype/dejavu/DejaVuSans.ttf")


def gen_text_phantom(recon_shape, words, font_size, font_path="DejaVuSans.ttf"):
    """utilities.py:750-825: each word rendered in a TrueType font, binarised, rotated onto the (col, slice) plane
    and written into one recon row; the rows are evenly spaced (row = Nr // (len(words) + 1) * (i + 1)) and the
    words centred in columns and slices.  Needs PIL and a font (font_path, else the reference's fallback paths);
    FileNotFoundError when there is none."""
    from PIL import Image, ImageDraw, ImageFont
    try:
        font = ImageFont.truetype(font_path, size=font_size)
    except OSError:
        for path in _FALLBACK_FONTS:
            if os.path.exists(path):
                font = ImageFont.truetype(path, size=font_size)
                break
        else:
            raise FileNotFoundError('Could not find a usable font. Tried the following paths:\n' +
                                    '\n'.join(_FALLBACK_FONTS) +
                                    '\nPlease install one of these fonts or specify a valid font_path.')
    nr, nc, ns = recon_shape
    size = int(min(nc, ns))
    phantom = np.zeros(recon_shape, dtype=np.float32)
    for i, word in enumerate(words):
        r, c, s = nr // (len(words) + 1) * (i + 1), nc // 2, ns // 2
        img = Image.new('L', (size, size), 0)
        draw = ImageDraw.Draw(img)
        left, top, right, bottom = draw.textbbox((0, 0), word, font=font)
        draw.text(((size - (right - left)) // 2 - left, (size - (bottom - top)) // 2 - top), word, fill=1, font=font)
        glyphs = (np.array(img.rotate(-90, expand=True).transpose(Image.FLIP_LEFT_RIGHT)) > 0).astype(np.float32)
        c0 = max(0, c - size // 2)
        c1 = min(nc, c0 + size)
        s0 = max(0, s - size // 2)
        s1 = min(ns, s0 + size)
        phantom[max(0, r):min(nr, r + 1), c0:c1, s0:s1] = glyphs[:c1 - c0, :s1 - s0]
    return phantom


def add_noise(sinogram, rel_sigma, seed):
    """sinogram + N(0, (rel_sigma * max|sinogram|)^2), seeded."""
    g = torch.Generator(device=sinogram.device).manual_seed(int(seed) + 1000)
    sigma = float(rel_sigma) * float(sinogram.abs().max())
    return sinogram + sigma * torch.randn(sinogram.shape, generator=g, device=sinogram.device, dtype=sinogram.dtype)


def uniform_angles(num_views, full_circle=False):
    stop = 2 * np.pi if full_circle else np.pi
    return np.linspace(0, stop, num_views, endpoint=False).astype(np.float32)


def batched_scan_shapes(num_scans=24):
    """Per-scan (views, det_rows, det_channels) of the uneven parallel-beam batch: scan i draws from seed i
    views U{60..720}, det_rows U{8..64}, det_channels U{96..512}."""
    shapes = []
    for i in range(num_scans):
        rng = np.random.default_rng(i)
        shapes.append((int(rng.integers(60, 721)), int(rng.integers(8, 65)), int(rng.integers(96, 513))))
    return shapes


def gen_translation_vectors(num_x_translations, num_z_translations, x_spacing, z_spacing):
    """(num_x * num_z, 3) translation vectors [dx, 0, dz] on a raster centred at 0, x fastest
    (utilities.py:1003-1031 of the reference)."""
    x = (np.arange(num_x_translations) - (num_x_translations - 1) / 2) * x_spacing
    z = (np.arange(num_z_translations) - (num_z_translations - 1) / 2) * z_spacing
    out = np.zeros((num_x_translations * num_z_translations, 3))
    out[:, 0] = np.tile(x, num_z_translations)
    out[:, 2] = np.repeat(z, num_x_translations)
    return out


def _h5py():
    try:
        import h5py
    except ImportError as e:
        raise ImportError('HDF5 files need the h5py package, which is not installed') from e
    return h5py


def save_data_hdf5(file_path, array, array_name='array', attributes_dict=None):
    """One dataset holding the array, with the entries of attributes_dict (converted to strings as
    TomographyModel.convert_subdicts_to_strings does) as its attributes (utilities.py:98-141 of the reference)."""
    h5py = _h5py()
    d = os.path.dirname(str(file_path))
    if d:
        os.makedirs(d, exist_ok=True)
    with h5py.File(file_path, 'w') as f:
        data = f.create_dataset(array_name, data=np.asarray(
            array.detach().cpu().numpy() if isinstance(array, torch.Tensor) else array))
        if isinstance(attributes_dict, dict):
            from .tomography_model import TomographyModel
            for key, value in TomographyModel.convert_subdicts_to_strings(attributes_dict).items():
                data.attrs[key] = value


def load_data_hdf5(file_path):
    """(array, attribute dict) from a file written by save_data_hdf5 (utilities.py:27-61 of the reference)."""
    h5py = _h5py()
    with h5py.File(file_path, 'r') as f:
        names = list(f.keys())
        if len(names) > 1:
            raise ValueError('More than one array found in {}. Unable to load.'.format(file_path))
        data = f[names[0]]
        array = data[()]
        data_dict = {name: data.attrs[name] for name in data.attrs.keys()}
    return array, data_dict
