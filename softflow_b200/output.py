"""Output and restart of a channel's state: the reference's writers
(src/io/vtk_writer.cpp, global_stats_writer.cpp, csv_writer.cpp,
fluid_probe_writer.cpp) and its binary checkpoint (src/io/checkpoint.cpp),
fed from the device state.

Nothing is mirrored on the host between steps: each writer pulls what it
needs at the call (the VTK writers inside the library, in C++; the
statistics from the device reductions of ``sfg_thermo``), so a run pays for
output only at the steps that write.  File names, column order and number
formatting follow the reference, so scripts that read its output read these
files unchanged.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
from typing import List, Optional

import numpy as np

from . import _lib as L

# FluidOutputFields defaults (io/output_config.h:10-21)
VTK_DENSITY, VTK_VELOCITY, VTK_VELOCITY_MAG, VTK_PRESSURE = 1, 2, 4, 8
VTK_VORTICITY, VTK_STRAIN_RATE, VTK_IBM_FORCE, VTK_NODE_TYPE = 16, 32, 64, 128
VTK_CONCENTRATION = 256
VTK_DEFAULT = (VTK_DENSITY | VTK_VELOCITY | VTK_VELOCITY_MAG | VTK_PRESSURE | VTK_NODE_TYPE |
               VTK_CONCENTRATION)


def _ctx(sim):
    return sim._need()


class VTKWriter:
    """Reference VTKWriter (vtk_writer.h:15-70): XML ImageData / PolyData
    files, or legacy .vtk files with ``legacy=True`` (the reference's
    vtk_format "legacy"), and the .pvd time-series collections."""

    def __init__(self, output_dir: str, legacy: bool = False, fields: int = VTK_DEFAULT):
        self.output_dir = output_dir
        self.legacy = bool(legacy)
        self.fields = int(fields)
        self._steps: List[int] = []
        self._times: List[float] = []
        os.makedirs(output_dir, exist_ok=True)

    def setLegacyMode(self, legacy: bool):
        self.legacy = bool(legacy)

    def writeFluidField(self, sim, step: int, chan: int = 0):
        ctx = _ctx(sim)
        L.check(ctx._lib.sfg_write_vtk_fluid(ctx._h, chan, self.output_dir.encode(), int(step),
                                             int(self.legacy), self.fields))

    def writeCapsules(self, sim, step: int, chan: int = 0):
        ctx = _ctx(sim)
        types = sim._chans[chan].caps
        tids = (C.c_int * max(len(types), 1))(*[r.type_id for r in types])
        L.check(ctx._lib.sfg_write_vtk_capsules(ctx._h, chan, self.output_dir.encode(),
                                                int(step), int(self.legacy), tids))

    def recordTimestep(self, step: int, time: float):
        self._steps.append(int(step))
        self._times.append(float(time))

    def writePVDFiles(self):
        """vtk_writer.cpp:473-547."""
        if not self._steps:
            return
        if self.legacy:
            pairs = [(os.path.join(self.output_dir, "fluid.pvd"), "fluid_%06d.vtk"),
                     (os.path.join(self.output_dir, "particles.pvd"), "particles_%06d.vtk")]
        else:
            pairs = [(os.path.join(self.output_dir, "fluid", "fluid.pvd"), "fluid_%06d.vti"),
                     (os.path.join(self.output_dir, "particles", "particles.pvd"),
                      "particles_%06d.vtp")]
        for path, pattern in pairs:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as fh:
                fh.write('<?xml version="1.0"?>\n')
                fh.write('<VTKFile type="Collection" version="0.1">\n<Collection>\n')
                for st, t in zip(self._steps, self._times):
                    fh.write('<DataSet timestep="%.6e" file="%s"/>\n' % (t, pattern % st))
                fh.write("</Collection>\n</VTKFile>\n")


class GlobalStatsWriter:
    """Reference GlobalStatsWriter (global_stats_writer.cpp:41-124): one row
    of global_stats.csv per call, from the device reductions."""

    def __init__(self, output_dir: str):
        self.output_dir = output_dir
        os.makedirs(output_dir, exist_ok=True)
        self._fh = None
        self._header = False

    def writeTimestep(self, sim, step: int, time: float, chan: int = 0):
        t = sim.thermo(chan)
        has_scalar = sim.advectionDiffusion(chan) is not None
        if self._fh is None:
            self._fh = open(os.path.join(self.output_dir, "global_stats.csv"), "a")
        fh = self._fh
        if not self._header:
            fh.write("timestep,time,mean_rho,max_velocity,mean_velocity,"
                     "total_kinetic_energy,n_active_particles,"
                     "mean_deformation,max_deformation,min_rho,max_rho")
            if has_scalar:
                fh.write(",total_dissolved_mass,total_particle_mass,total_adsorbed_mass")
            fh.write("\n")
            self._header = True
        fh.write("%d,%.6e,%.6e,%.6e,%.6e,%.6e,%d,%.6e,%.6e,%.6e,%.6e" % (
            step, time, t["mean_rho"], t["max_speed"], t["mean_velocity"],
            t["kinetic_energy"], t["num_capsules"], t["mean_deformation"],
            t["max_deformation"], t["min_rho"], t["max_rho"]))
        if has_scalar:
            # no capsule chemistry on this path: reservoirs are infinite
            # (not counted) and nothing is adsorbed
            fh.write(",%.6e,%.6e,%.6e" % (t["total_scalar"], 0.0, 0.0))
        fh.write("\n")
        fh.flush()

    def close(self):
        if self._fh is not None:
            self._fh.close()
            self._fh = None


class CSVWriter:
    """Reference CSVWriter (csv_writer.cpp:8-154) with its default fields
    (type, centroid, mean node velocity): one row per capsule per call."""

    def __init__(self, output_dir: str, filename: str = "particle_data.csv",
                 fmt: str = "csv", append: bool = True):
        self.output_dir = output_dir
        self.path = os.path.join(output_dir, filename)
        self.sep = "\t" if fmt in ("dat", "DAT") else ","
        self.append = append
        os.makedirs(output_dir, exist_ok=True)
        self._fh = None
        self._header = False

    def writeTimestep(self, sim, step: int, time: float, chan: int = 0):
        if self._fh is None:
            self._fh = open(self.path, "a" if self.append else "w")
        s, fh = self.sep, self._fh
        if not self._header:
            fh.write(f"timestep{s}time{s}capsule_id{s}type{s}cx{s}cy{s}vx{s}vy\n")
            self._header = True
        caps = sim.capsules(chan)
        vel = caps.velocities()
        stats = sim._need().thermo()[1]
        base = caps._cap_base
        recs = sim._chans[chan].caps
        for c in range(caps.numCapsules()):
            o, n = caps._offsets[c], caps._counts[c]
            vx = vy = 0.0
            for k in range(o, o + n):
                vx += float(vel[k, 0])
                vy += float(vel[k, 1])
            vx /= n
            vy /= n
            cx, cy = stats[base + c, 0], stats[base + c, 1]
            fh.write("%d%s%.6e%s%d%s%d%s%.6e%s%.6e%s%.6e%s%.6e\n" % (
                step, s, time, s, c, s, recs[c].type_id, s, cx, s, cy, s, vx, s, vy))
        fh.flush()

    def close(self):
        if self._fh is not None:
            self._fh.close()
            self._fh = None


class FluidProbeWriter:
    """Reference FluidProbeWriter (fluid_probe_writer.cpp:8-73):
    rho, ux, uy, p at chosen cells into fluid_probes.csv."""

    def __init__(self, output_dir: str):
        self.output_dir = output_dir
        os.makedirs(output_dir, exist_ok=True)
        self.probes = []
        self._fh = None
        self._header = False

    def addProbe(self, i: int, j: int, label: str):
        self.probes.append((int(i), int(j), str(label)))
        self._header = False

    def writeTimestep(self, sim, step: int, time: float, chan: int = 0):
        if not self.probes:
            return
        if self._fh is None:
            self._fh = open(os.path.join(self.output_dir, "fluid_probes.csv"), "a")
        fh = self._fh
        if not self._header:
            fh.write("timestep,time")
            for _, _, lb in self.probes:
                fh.write(f",{lb}_rho,{lb}_ux,{lb}_uy,{lb}_p")
            fh.write("\n")
            self._header = True
        fld = sim.field(chan)
        rho, ux, uy, _, _ = fld.macroscopic()
        ny, nx = rho.shape
        fh.write("%d,%.6e" % (step, time))
        for i, j, _ in self.probes:
            x, y = min(max(i, 0), nx - 1), min(max(j, 0), ny - 1)
            r = float(rho[y, x])
            fh.write(",%.6e,%.6e,%.6e,%.6e" % (r, float(ux[y, x]), float(uy[y, x]), r / 3.0))
        fh.write("\n")
        fh.flush()

    def close(self):
        if self._fh is not None:
            self._fh.close()
            self._fh = None


# --------------------------------------------------------------- checkpoint
class CheckpointError(RuntimeError):
    pass


class Checkpoint:
    """The reference's binary checkpoint, version 4 (io/checkpoint.cpp:10-48,
    76-195 save, 197-371 load): "SFCK", version, step, nx, ny, ncaps; the
    populations f [9][ny][nx], rho, ux, uy, the cell types; per capsule id,
    type, node count, positions, velocities, current area and perimeter,
    periodic_nx; the adhesion bond count (0 here); the scalar block.  Native
    byte order and sizes (int32, float64), as the reference writes them."""

    VERSION = 4

    @staticmethod
    def save(sim, filename: str, chan: int = 0, step: Optional[int] = None) -> str:
        """step: the step number stored in the file (default: steps run)."""
        ctx = sim._need()
        p = sim._chans[chan].params
        nx, ny = p.nx, p.ny
        fld = sim.field(chan)
        f = fld.distributions()
        rho, ux, uy, _, _ = fld.macroscopic()
        flags = np.zeros((ny, nx), dtype=np.int32)
        if not p.fluid.periodic_y:
            flags[0, :] = 1
            flags[ny - 1, :] = 1
        caps = sim.capsules(chan)
        n = caps.numCapsules()
        pos, vel = (caps.positions(), caps.velocities()) if n else (None, None)
        stats = ctx.thermo()[1]
        base = caps._cap_base
        recs = sim._chans[chan].caps
        d = os.path.dirname(os.path.abspath(filename))
        os.makedirs(d, exist_ok=True)
        with open(filename, "wb") as fh:
            fh.write(b"SFCK")
            st = int(sim.currentStep() if step is None else step)
            fh.write(struct.pack("=iiiii", Checkpoint.VERSION, st, nx, ny, n))
            fh.write(np.ascontiguousarray(f, dtype=np.float64).tobytes())
            for a in (rho, ux, uy):
                fh.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
            fh.write(flags.tobytes())
            for c in range(n):
                o, nn = caps._offsets[c], caps._counts[c]
                fh.write(struct.pack("=iii", c, recs[c].type_id, nn))
                fh.write(np.ascontiguousarray(pos[o:o + nn], dtype=np.float64).tobytes())
                fh.write(np.ascontiguousarray(vel[o:o + nn], dtype=np.float64).tobytes())
                # the reference stores the current area and perimeter here
                fh.write(struct.pack("=ddi", float(stats[base + c, 2]),
                                     float(stats[base + c, 3]), nx))
            fh.write(struct.pack("=i", 0))                 # adhesion bonds
            ad = sim.advectionDiffusion(chan)
            fh.write(struct.pack("=i", 1 if ad is not None else 0))
            if ad is not None:
                fh.write(struct.pack("=i", 1))             # species
                g = ad.populations()                       # [9][ny][nx]
                # AdvectionDiffusion keeps g cell-major: g[n * 9 + q]
                fh.write(np.ascontiguousarray(g.reshape(9, -1).T).tobytes())
                fh.write(np.ascontiguousarray(ad.concentration(), dtype=np.float64).tobytes())
                fh.write(struct.pack("=i", 0))             # tracked capsules
                fh.write(struct.pack("=i", 0))             # reservoir masses
                fh.write(struct.pack("=i", 0))             # surface coverage
        return filename

    @staticmethod
    def load(sim, filename: str, chan: int = 0) -> int:
        """Restores a checkpoint into a freshly initialized simulation of the
        same geometry; returns the restored step.  As in the reference, the
        populations, marker positions and velocities and the scalar state
        are restored; rest state and membrane memory are those of the
        simulation (the Kelvin-Voigt term starts over)."""
        ctx = sim._need()
        if sim.currentStep() != 0:
            raise CheckpointError("load into a simulation that has not stepped yet")
        p = sim._chans[chan].params
        with open(filename, "rb") as fh:
            buf = fh.read()
        if buf[:4] != b"SFCK":
            raise CheckpointError("invalid magic (not a SoftFlow checkpoint)")
        off = 4
        (version,) = struct.unpack_from("=i", buf, off)
        off += 4
        if version < 2 or version > 4:
            raise CheckpointError(f"unsupported version {version} (expected 2, 3, or 4)")
        step, nx, ny, ncaps = struct.unpack_from("=iiii", buf, off)
        off += 16
        if nx != p.nx or ny != p.ny:
            raise CheckpointError(f"domain mismatch. File has {nx}x{ny} but simulation is "
                                  f"{p.nx}x{p.ny}")
        caps = sim.capsules(chan)
        if ncaps != caps.numCapsules():
            raise CheckpointError(f"capsule count mismatch. File has {ncaps} but simulation "
                                  f"has {caps.numCapsules()}")
        N = nx * ny

        def take(count, dtype):
            nonlocal off
            a = np.frombuffer(buf, dtype=dtype, count=count, offset=off)
            off += a.nbytes
            return a

        f = take(9 * N, np.float64).copy()
        take(3 * N, np.float64)          # rho, ux, uy: recomputed from f and the body force
        take(N, np.int32)                # cell types: fixed by the channel geometry
        pos = np.zeros((caps.totalNodes(), 2))
        vel = np.zeros((caps.totalNodes(), 2))
        for c in range(ncaps):
            _, _, nn = struct.unpack_from("=iii", buf, off)
            off += 12
            if nn != caps._counts[c]:
                raise CheckpointError(f"node count mismatch for capsule {c}. File has {nn}, "
                                      f"sim has {caps._counts[c]}")
            o = caps._offsets[c]
            pos[o:o + nn] = take(2 * nn, np.float64).reshape(nn, 2)
            vel[o:o + nn] = take(2 * nn, np.float64).reshape(nn, 2)
            off += 8 + 8 + 4             # saved area, perimeter, periodic_nx
        (nbonds,) = struct.unpack_from("=i", buf, off)
        off += 4 + nbonds * (4 * 4 + 2 * 8)
        scalar = None
        if version >= 3:
            (has_scalar,) = struct.unpack_from("=i", buf, off)
            off += 4
            ad = sim.advectionDiffusion(chan)
            if has_scalar and ad is not None:
                (ns,) = struct.unpack_from("=i", buf, off)
                off += 4
                if ns != 1:
                    raise CheckpointError(f"scalar species count mismatch. File has {ns}, "
                                          "sim has 1")
                g = take(9 * N, np.float64).reshape(N, 9).T.copy()
                Cf = take(N, np.float64).copy()
                scalar = (Cf, g)
        fld = sim.field(chan)
        fld.set_distributions(f)
        if ncaps:
            caps.set_state(pos, vel)
        if scalar is not None:
            L.check(ctx._lib.sfg_set_scalar_state(ctx._h, chan, L.dptr(scalar[0]),
                                                  L.dptr(scalar[1])))
        L.check(ctx._lib.sfg_mark_restored(ctx._h))
        ctx.touch()
        sim._steps = int(step)
        return int(step)
