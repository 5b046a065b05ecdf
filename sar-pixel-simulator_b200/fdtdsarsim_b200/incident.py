"""Incident-beam generation on the device.

The reference makes the beam of a geometry on the CPU in three stages
(IncidentBeam.setup, incidentbeam.py:41-71): a Gaussian-tapered complex
carrier (create_pulse, :174-204), its lateral excitation as a tapered wave
(create_inc_excitation, :206-298), and a vacuum FDTD run that injects the
excitation as a hard source and records the fields on a read-out plane
(IncidentSimCpu, cpu/incident_sim.py:22-171). The pulse is a 1-D array and
stays on the host here; the excitation (two (size_t_inc, ny, nx) complex
arrays) and the run are computed by libfdtd_b200 without a host round trip
(fdtd_incident_make_excitation, fdtd_incident_run). The recorded planes are
written to the incident file in the reference's layout, and can also be
handed to a main simulation on the device (NativeSim.set_incident_from).
"""
import copy
import logging
import os
import threading

import numpy as np
import scipy.constants

from . import _native
from .absorbers import packed_profiles
from .parameters import ParameterCollection, inc_filename

logger = logging.getLogger(__name__)


def create_pulse(params: ParameterCollection):
    """(time_vals, pulse, pulse_fft, pulse_freqs): the Gaussian-tapered
    complex carrier of incidentbeam.py:174-199 and its spectrum. The
    duration is the time at which the Gaussian falls to a tenth of its
    peak."""
    g, inc = params.geom_params, params.inc_beam_params
    dt, nt_inc, nt_pulse = g.timestep, g.size_t_inc, g.size_t_pulse
    time_vals = np.linspace(0.0, dt * (nt_inc - 1), num=nt_inc, endpoint=True)
    sig = inc.duration / inc.frequency / (2.0 * np.sqrt(2.0 * np.log(10.0)))
    om = 2.0 * np.pi * inc.frequency
    pulse = 1.0 * np.exp(-(time_vals - (dt * nt_pulse / 2)) ** 2 / (sig ** 2)) * np.exp(1j * om * time_vals)
    return time_vals, pulse, np.fft.fft(pulse), np.fft.fftfreq(pulse.size, dt)


def taper_radius(params: ParameterCollection):
    """Radius of the beam's Gaussian footprint: the illumination width (in
    wavelengths) is where the taper falls to a tenth (incidentbeam.py:
    228-233)."""
    inc = params.inc_beam_params
    width = inc.illumination_width * scipy.constants.c / inc.frequency
    return width / (2.0 * np.sqrt(2.0 * np.log(10.0)))


def incident_params(params: ParameterCollection) -> ParameterCollection:
    """The parameters of the incident run: the geometry's, with the grid
    height fixed to 3 wavelengths (cpu/incident_sim.py:33-37)."""
    p = copy.deepcopy(params)
    lam = scipy.constants.c / p.inc_beam_params.frequency
    p.geom_params.size_z = int(3.0 * lam / p.geom_params.cell_size)
    return p


class IncidentSimGpu:
    """The incident-beam simulation of one geometry on the device
    (counterpart of IncidentSimCpu, cpu/incident_sim.py:22-171)."""

    def __init__(self, params: ParameterCollection, device: int = 0):
        from .gpu.main_sim import native_geometry
        self.params = incident_params(params)
        g = self.params.geom_params
        geom = native_geometry(self.params)
        geom.nt = g.size_t_inc
        geom.nt_inc = 0
        geom.tfsf_z = g.size_z // 2
        self.native = _native.NativeIncident(geom, g.size_t_pulse, device)
        self.native.set_absorbers(packed_profiles(self.params))
        self.peak = None

    def make_excitation(self, pulse_fft, pulse_freqs):
        """The excitation of create_inc_excitation on the device, from the
        pulse spectrum; returns the peak magnitude it normalised to 10."""
        inc = self.params.inc_beam_params
        k_vals = (2 * np.pi * np.asarray(pulse_freqs, dtype=np.float64)) / scipy.constants.c
        self.peak = self.native.make_excitation(k_vals, pulse_fft, inc.theta_angle, inc.phi_angle,
                                                inc.polarization, taper_radius(self.params))
        return self.peak

    def set_excitation(self, pulse_ex, pulse_ey):
        """Use a given excitation instead: the reference's complex
        (size_t_inc, ny, nx) arrays, of which the run injects the imaginary
        parts of the first size_t_pulse samples (cpu/incident_sim.py:
        108-110,141-144), or those imaginary parts themselves as real arrays
        (what IncidentBeam.create_inc_excitation returns)."""
        n = self.native.nt_pulse
        pick = (lambda a: np.imag(a)[:n]) if np.iscomplexobj(pulse_ex) else (lambda a: np.asarray(a)[:n])
        self.native.set_excitation(pick(pulse_ex), pick(pulse_ey))

    def run(self, pulse_ex=None, pulse_ey=None):
        """Run the beam simulation; with no arguments, on the excitation
        already set or made on the device."""
        if pulse_ex is not None:
            self.set_excitation(pulse_ex, pulse_ey)
        self.native.run()

    def planes(self):
        """The recorded ex, ey, hx, hy planes, (size_t_inc, ny, nx) each."""
        return self.native.get_planes()

    def phasors(self):
        """{ex,ey,hx,hy}_inc_phasor of the read-out plane."""
        return self.native.get_phasors()

    def close(self):
        self.native.close()


# Incident runs just made by IncidentBeam.setup, kept on the device for the
# next main simulation of the same geometry: {absolute incident file name:
# (IncidentSimGpu, phasors)}. MainSimGpu takes an entry (device-to-device
# copy of the planes, then the run is closed) instead of reading the file
# back; the file is still written, for other processes and later runs.
_RESIDENT = {}


def keep_resident(fname: str, sim: 'IncidentSimGpu', phasors):
    """Hold an incident run for the next main simulation that needs its
    file (replacing any run held for that file)."""
    import os
    key = os.path.abspath(fname)
    old = _RESIDENT.pop(key, None)
    if old is not None:
        old[0].close()
    _RESIDENT[key] = (sim, phasors)


def take_resident(fname: str):
    """(IncidentSimGpu, phasors) held for an incident file, or None; the
    caller closes the run."""
    import os
    return _RESIDENT.pop(os.path.abspath(fname), None)


def make_incident_beam(params: ParameterCollection, device=None):
    """The incident beam of a geometry made on the device: (planes, phasors,
    sim), the recorded planes and incident phasors as host arrays and the
    IncidentSimGpu (still holding the planes on the device, for
    NativeSim.set_incident_from; close it when done)."""
    from .gpu.main_sim import _device_of
    dev = _device_of(params) if device is None else int(device)
    _, _, pulse_fft, pulse_freqs = create_pulse(params)
    sim = IncidentSimGpu(params, dev)
    sim.make_excitation(pulse_fft, pulse_freqs)
    sim.run()
    return sim.planes(), sim.phasors(), sim


def generate_incident_beam(params: ParameterCollection, write: bool = True, device=None):
    """make_incident_beam and, with ``write``, the incident file in the
    reference's layout, written before returning."""
    planes, phasors, sim = make_incident_beam(params, device)
    if write:
        store_incident_beam(params, planes, phasors)
    return planes, phasors, sim


# Incident files being written on a thread: {absolute file name: thread}.
# Readers in this process wait for the write (wait_written); the threads are
# not daemons, so the interpreter also waits for them before it exits.
_WRITES = {}
_WRITES_LOCK = threading.Lock()


def store_incident_beam(params: ParameterCollection, planes, phasors, background: bool = False):
    """Write the incident file of a beam (and check it as IncidentBeam.setup
    checks a new file, incidentbeam.py:57-62); with ``background`` on a
    thread, so that the device can go on while the file is written."""
    from .incidentbeam import IncidentBeam, write_incident_file
    pc = copy.deepcopy(params)

    def write():
        write_incident_file(pc, planes['ex'], planes['ey'], planes['hx'], planes['hy'], phasors)
        IncidentBeam(pc).check_file()

    fname = os.path.abspath(inc_filename(pc))
    wait_written(fname)                  # one writer per file at a time
    if not background:
        write()
        return
    errors = []

    def run():
        try:
            write()
        except BaseException as exc:   # handed to the thread that waits
            errors.append(exc)

    t = threading.Thread(target=run, name='incident-file-write')
    t.errors = errors
    with _WRITES_LOCK:   # a waiter never finds an entry whose thread has not started
        _WRITES[fname] = t
        t.start()


def wait_written(fname=None):
    """Wait for the background write of incident file ``fname`` (of every
    such write when None) and raise the first error one of them met. Every
    waiter that finds a write in progress blocks until it ends and sees its
    error; the entry is removed only after the write has ended."""
    with _WRITES_LOCK:
        keys = [os.path.abspath(fname)] if fname is not None else list(_WRITES)
        found = [(key, _WRITES.get(key)) for key in keys]
    first = None
    for key, t in found:
        if t is None:
            continue
        t.join()
        with _WRITES_LOCK:
            if _WRITES.get(key) is t:
                del _WRITES[key]
        if t.errors and first is None:
            first = t.errors[0]
    if first is not None:
        raise first
