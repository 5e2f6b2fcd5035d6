"""Writes c2_spheres_512.params: the 512^3 precision-study solve -- 20 nm uniform grid,
12-cell CPML, 4000 dielectric spheres with seeded random centres (uniform in the core box),
radii (uniform in 3..12 cells) and permittivities (uniform in 2..12), later spheres over
earlier ones; z dipole (Gaussian-modulated sine, 193.4 THz, 50 THz FWHM) at core cell
(160, 256, 256); Ez probe at (352, 256, 256) + 21-frequency DFT.  Seed 2 (numpy PCG64), so
the file is reproducible: `python make_c2_spheres.py > c2_spheres_512.params`."""
import numpy as np

N, D = 512, 20e-9
L = N * D
rng = np.random.default_rng(2)
c = rng.uniform(0.0, L, size=(4000, 3))
r = rng.uniform(3.0, 12.0, size=4000) * D
eps = rng.uniform(2.0, 12.0, size=4000)
head = f"""# 512^3 precision study: 4000 seeded random dielectric spheres in vacuum (written by
# make_c2_spheres.py, seed 2), 20 nm uniform grid, 12-cell CPML (536^3 total cells),
# z dipole as in the 64^3 case at core cell (160, 256, 256), Ez probe + 21-frequency DFT.
MESH_MODE = 0
NX = {N}
NY = {N}
NZ = {N}
DX_UNIFORM = {D}
DY_UNIFORM = {D}
DZ_UNIFORM = {D}
DOMAIN_X_MIN = 0
DOMAIN_X_MAX = {L}
DOMAIN_Y_MIN = 0
DOMAIN_Y_MAX = {L}
DOMAIN_Z_MIN = 0
DOMAIN_Z_MAX = {L}
LAMBDA0 = 1550.1264633919338e-9
CFL_FACTOR = 0.99
N_STEPS = 5000
SAVE_EVERY = 1
CPML_NPML = 12
CPML_M = 3.0
CPML_RERR = 1e-6
CPML_ALPHA0 = 0.05
CPML_KAPPA_MAX = 5.0
CPML_ALPHA_LINEAR = true
BACKGROUND_N = 1.0
TLS_ENABLED = false
MESH_OVERRIDE_ENABLED = false
DIPOLE_SOURCES += true, {160.5 * D}, {256.5 * D}, {256.5 * D}, 1e-7, 193.4e12, 0, 0, 50e12, 3.0, 1, 2
POINT_FIELD_DETECTORS += true, Ez_probe, {352.5 * D}, {256.5 * D}, {256.5 * D}, 2
DFT_FREQS = 168e12, 218e12, 21
PRECISION = fp32"""
print(head)
for k in range(4000):
    print(f"STRUCTURES += sphere, {np.sqrt(eps[k]):.17g}, {c[k,0]:.17g}, {c[k,1]:.17g}, {c[k,2]:.17g}, {r[k]:.17g}, 0, 0, \"\"")
