"""Reference input files for the oracle harness (test infrastructure only).

Text of VAMPIRE `input` and material files (the reference's own
"key:word=value !unit" format, src/vio/match.cpp:72-83) for the synthetic
benchmark systems: simple-cubic and FCC boxes with nearest-neighbour exchange,
uniaxial or cubic anisotropy, and the two-material A/B alloy with DMI.
"""


def sc_input(L: int, a: float = 3.0, T: float = 0.0, H: float = 0.1, periodic: bool = True,
             integrator: str = "llg-heun", extra: str = "") -> str:
    size = L * a / 10.0
    pb = "".join(f"create:periodic-boundaries-{c}\n" for c in "xyz") if periodic else ""
    return (f"create:crystal-structure=sc\n{pb}dimensions:unit-cell-size={a} !A\n"
            f"dimensions:system-size-x={size} !nm\ndimensions:system-size-y={size} !nm\n"
            f"dimensions:system-size-z={size} !nm\nmaterial:file=m.mat\nsim:temperature={T}\n"
            f"sim:time-step=1.0E-16\nsim:applied-field-strength={H} !T\n"
            f"sim:applied-field-unit-vector=0,0,1\nsim:program=time-series\n"
            f"sim:integrator={integrator}\n{extra}")


SC_MAT = """material:num-materials=1
material[1]:material-name=A
material[1]:damping-constant=0.1
material[1]:exchange-matrix[1]=11.2e-21
material[1]:atomic-spin-moment=1.72 !muB
material[1]:second-order-uniaxial-anisotropy-constant=6.69e-24
material[1]:uniaxial-anisotropy-direction=0,0,1
material[1]:initial-spin-direction=random
"""


def fcc_input(L: int, T: float = 300.0, extra: str = "") -> str:
    a = 3.54
    size = L * a / 10.0
    return (f"create:crystal-structure=fcc\n" + "".join(f"create:periodic-boundaries-{c}\n" for c in "xyz") +
            f"dimensions:unit-cell-size={a} !A\ndimensions:system-size-x={size} !nm\n"
            f"dimensions:system-size-y={size} !nm\ndimensions:system-size-z={size} !nm\n"
            f"material:file=m.mat\nsim:temperature={T}\nsim:time-step=1.0E-16\n"
            f"sim:program=time-series\nsim:integrator=llg-heun\n{extra}")


def fcc_mat(J_AA=11.2e-21, J_AB=5.0e-21, Kc=1.0e-24, alpha=0.05) -> str:
    out = ["material:num-materials=2"]
    for i, (name, jself, jother) in enumerate([("A", J_AA, J_AB), ("B", J_AA, J_AB)], start=1):
        other = 2 if i == 1 else 1
        out += [f"material[{i}]:material-name={name}",
                f"material[{i}]:damping-constant={alpha}",
                f"material[{i}]:exchange-matrix[{i}]={jself}",
                f"material[{i}]:exchange-matrix[{other}]={jother}",
                f"material[{i}]:dmi-constant[{i}]={0.1 * jself}",
                f"material[{i}]:dmi-constant[{other}]={0.1 * jother}",
                f"material[{i}]:atomic-spin-moment=1.72 !muB",
                f"material[{i}]:fourth-order-cubic-anisotropy-constant={Kc}",
                f"material[{i}]:initial-spin-direction=random"]
    out += ["material[1]:host-alloy", "material[1]:alloy-fraction[2]=0.5"]
    return "\n".join(out) + "\n"
