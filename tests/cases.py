"""Small configurations used by the parity tests (odd sizes, every boundary
type, 2D and 3D)."""
import ifc


def small_cases():
    cav = ifc.cavity2d(17, ny=13)
    chan = ifc.channel2d(20, 9)
    mixed = ifc.channel2d(12, 11)
    mixed["velBC_type"] = [ifc.OUTLET, ifc.INLET, ifc.INLET, ifc.WALL, ifc.WALL, ifc.WALL]
    mixed["velBC_val"] = [[0, 0, 0], [0.002, 0.0005, 0], [0.0003, -0.001, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0]]
    cav3 = ifc.cavity3d(6, nx=6, ny=5, nz=4)
    chan3 = ifc.cavity3d(7, nx=7, ny=5, nz=6, density=3.0, dynamicViscosity=0.05)
    chan3["velBC_type"] = [ifc.OUTLET, ifc.INLET, ifc.WALL, ifc.WALL, ifc.WALL, ifc.OUTLET]
    chan3["velBC_val"] = [[0, 0, 0], [0.7, 0.1, -0.2], [0, 0, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0]]
    for c in (cav, chan, mixed, cav3, chan3):
        c["nIter_p"] = 7
        c["nIter_u"] = c["nIter_v"] = c["nIter_w"] = 3
    return {"cavity17x13": cav, "channel20x9": chan, "mixed12x11": mixed,
            "cavity6x5x4": cav3, "channel7x5x6": chan3}
