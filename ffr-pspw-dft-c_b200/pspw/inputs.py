"""Writers of input files in the reference's own formats: an INPUT keyword
file (the keywords ReadInputFile.cpp:37-186 reads) and a synthetic
norm-conserving pseudopotential in the FHI98 layout ReadPseudopotentials.cpp
reads.  Used to run the reference program and the engine on the same
inputs."""
from __future__ import annotations


def write_synthetic_fhi(path, zv=4.0, well=1.0, width=1.2):
    """A synthetic norm-conserving pseudopotential in the FHI98 text layout
    the reference reads (ReadPseudopotentials.cpp:27-62): `ZV nang`, ten
    skipped lines, then per angular momentum `mmax clog` and mmax rows
    `i r u(r) V(r)` on a logarithmic mesh.  The model: V_loc = -ZV erf(r)/r
    + well exp(-(r/width)^2) (a negative `well` is an attractive Gaussian
    of depth -well), V_s = V_loc + 1.5 exp(-(r/0.9)^2),
    V_p = V_loc - 0.7 exp(-(r/1.1)^2), V_d = V_loc; u_l(r) = r^(l+1)
    exp(-r^2/4) normalised."""
    from math import erf, exp, sqrt
    mmax, r1, fac = 495, 4.5e-4, 1.0247
    rs = [r1 * fac ** i for i in range(mmax)]

    def vloc(r):
        return -zv * erf(r) / r + well * exp(-(r / width) ** 2)

    def vl(l, r):
        if l == 0:
            return vloc(r) + 1.5 * exp(-(r / 0.9) ** 2)
        if l == 1:
            return vloc(r) - 0.7 * exp(-(r / 1.1) ** 2)
        return vloc(r)

    lines = [f"{zv:.5E}    3"] + [" 0.0000    .00e+00   .00e+00"] * 10
    h = (fac - 1.0)
    for l in range(3):
        u = [r ** (l + 1) * exp(-r * r / 4.0) for r in rs]
        norm = sqrt(sum(x * x * r for x, r in zip(u, rs)) * h)
        lines.append(f"{mmax}  {fac:.14E}")
        for i, r in enumerate(rs):
            lines.append(f"{i + 1:4d} {r:.14E} {u[i] / norm:.14E} {vl(l, r):.14E}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_input(path, fhi_name, positions, a, ecut_ry=8.0, iscf=1, idiag=0, imix=2,
                max_scf=40, nempty=5, fft_grid=None, conv=None, degree=None):
    """An INPUT file in the reference's keyword format (ReadInputFile.cpp):
    one species of len(positions) atoms in a cubic cell of side a (bohr)."""
    pos = "\n".join(f"  {p[0]:.9f} {p[1]:.9f} {p[2]:.9f}" for p in positions)
    txt = (f"iscf\n {iscf}\n\nidiag\n {idiag}\n\nimix\n {imix}\n\nrho_mix_fac\n 0.3\n\n"
           f"max_scf_iter\n {max_scf}\n\nnempty\n {nempty}\n\necut\n {ecut_ry}\n\n"
           f"atoms\n 1\n {len(positions)}\n {fhi_name}\n 3 3\n bohr\n{pos}\n\n"
           f"latvec\n {a} 0.0 0.0\n 0.0 {a} 0.0\n 0.0 0.0 {a}\n\n"
           f"k_points\n 1\n 0.0 0.0 0.0 1.0\n")
    if fft_grid is not None:
        txt += f"\nfft_grid\n {fft_grid[0]} {fft_grid[1]} {fft_grid[2]}\n"
    if conv is not None:
        txt += f"\nscf_conv_crit\n {conv:.6e}\n"
    if degree is not None:
        txt += f"\nchebypol_degree\n {degree}\n"
    with open(path, "w") as f:
        f.write(txt)


def write_input_species(path, species, a, ecut_ry, nempty, fft_grid=None, imix=3, idiag=-1,
                        max_scf=100, conv=None, degree=None, ekt=None):
    """An INPUT file with several species in a cubic cell of side a (bohr):
    species = [(fhi_name, positions (n, 3) in bohr), ...], in the atoms
    block layout ReadInputFile.cpp:53-92 reads (NSP; NA per species; per
    species the file, `LMAX LLOC`, the coordinate type and NA lines).
    ekt (eV) adds `tmetal .true.` and `ekt` (ReadInputFile.cpp:116-125)."""
    nas = " ".join(str(len(p)) for _, p in species)
    blocks = []
    for name, pos in species:
        lines = "\n".join(f"  {p[0]:.9f} {p[1]:.9f} {p[2]:.9f}" for p in pos)
        blocks.append(f" {name}\n 3 3\n bohr\n{lines}")
    txt = (f"iscf\n 1\n\nidiag\n {idiag}\n\nimix\n {imix}\n\nrho_mix_fac\n 0.3\n\n"
           f"max_scf_iter\n {max_scf}\n\nnempty\n {nempty}\n\necut\n {ecut_ry}\n\n"
           f"atoms\n {len(species)}\n {nas}\n" + "\n".join(blocks) + "\n\n"
           f"latvec\n {a} 0.0 0.0\n 0.0 {a} 0.0\n 0.0 0.0 {a}\n\n"
           f"k_points\n 1\n 0.0 0.0 0.0 1.0\n")
    if fft_grid is not None:
        txt += f"\nfft_grid\n {fft_grid[0]} {fft_grid[1]} {fft_grid[2]}\n"
    if conv is not None:
        txt += f"\nscf_conv_crit\n {conv:.6e}\n"
    if degree is not None:
        txt += f"\nchebypol_degree\n {degree}\n"
    if ekt is not None:
        txt += f"\ntmetal\n .true.\n\nekt\n {ekt}\n"
    with open(path, "w") as f:
        f.write(txt)
