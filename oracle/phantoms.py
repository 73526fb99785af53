"""CPU restatement of the reference's brain phantom and dataset-generator mask.

TEST INFRASTRUCTURE ONLY: tests compare the device rasteriser
(ceep_b200.dataset / ceep_brain_phantom_2d) with these functions; the product
never imports this module.

* brain_phantom_maps  - BrainPhantom2D.get_eps_map with the fixed tissue table
                        (src/ceep/phantoms/head_models.py:519-631,
                        use_gabriel_database=False)
* hemorrhage_mask     - scripts/generate_corrected_dataset.py:110-118

Pinned to tests/golden/brain_phantom.npz (made by the reference's own class).
"""
from __future__ import annotations

import numpy as np

# head_models.py:583-590 (eps_r, sigma) and layer thicknesses :538-541
TISSUE = {"skin": (40.0, 1.0), "skull": (12.0, 0.2), "csf": (68.0, 2.5), "gray": (52.0, 1.8),
          "white": (38.0, 1.2), "blood": (61.0, 2.0)}
THICKNESS = {"skin": 3e-3, "skull": 7e-3, "csf": 2e-3, "gray": 10e-3}


def layer_radii(head_radius_cm: float):
    """Outer radii (m) of skin, skull, csf, grey, white (head_models.py:600-604)."""
    r_skin = head_radius_cm * 1e-2
    r_skull = r_skin - THICKNESS["skin"]
    r_csf = r_skull - THICKNESS["skull"]
    r_gray = r_csf - THICKNESS["csf"]
    r_white = r_gray - THICKNESS["gray"]
    return r_skin, r_skull, r_csf, r_gray, r_white


def brain_phantom_maps(nx, ny, dx, hemorrhage_location=None, hemorrhage_radius_cm=1.0, head_radius_cm=9.0):
    eps = np.ones((nx, ny))
    sig = np.zeros((nx, ny))
    cx, cy = nx // 2, ny // 2
    xg, yg = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    r = np.sqrt(((xg - cx) * dx) ** 2 + ((yg - cy) * dx) ** 2)
    r_skin, r_skull, r_csf, r_gray, r_white = layer_radii(head_radius_cm)
    for mask, name in (((r <= r_skin) & (r > r_skull), "skin"), ((r <= r_skull) & (r > r_csf), "skull"),
                       ((r <= r_csf) & (r > r_gray), "csf"), ((r <= r_gray) & (r > r_white), "gray"),
                       (r <= r_white, "white")):
        eps[mask], sig[mask] = TISSUE[name]
    if hemorrhage_location is not None:
        hx, hy = hemorrhage_location[0] * 1e-2, hemorrhage_location[1] * 1e-2
        rh = np.sqrt(((xg - cx) * dx - hx) ** 2 + ((yg - cy) * dx - hy) ** 2)
        m = rh <= hemorrhage_radius_cm * 1e-2
        eps[m], sig[m] = TISSUE["blood"]
    return eps, sig


def hemorrhage_mask(nx, ny, dx, hemorrhage_location, hemorrhage_radius_cm):
    mask = np.zeros((nx, ny))
    if hemorrhage_location is None:
        return mask
    cx, cy = nx // 2, ny // 2
    xg, yg = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    r = np.sqrt(((xg - cx) * dx - hemorrhage_location[0] * 1e-2) ** 2
                + ((yg - cy) * dx - hemorrhage_location[1] * 1e-2) ** 2)
    mask[r <= hemorrhage_radius_cm * 1e-2] = 1.0
    return mask
