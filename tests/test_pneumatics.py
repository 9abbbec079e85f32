"""Pneumatic port mass flows on the device (swb_port_mass_flows) against the
reference's evaluateOrificeMassFlow / evaluateConductanceMassFlow
(pneumatics.cpp:132-232), compiled into oracle/_ref.

The conductance law is plain arithmetic and must match byte for byte.  The
orifice law raises ratios to non-integer powers; CUDA's double pow and the
host C library's may differ in the last bits, and the subsonic law
subtracts two such powers, which near equal pressures amplifies those bits
by 1 / (1 - ratio).  Orifice flows are therefore compared to 1e-12
relative, with most of them (86 %) exact, and the flow direction and the choked
flag must agree exactly.  Every
refusal of the reference is reported at the same port.
"""
import numpy as np
import pytest

import simwing_b200 as sw
import simwing_b200.abi as abi
from oracle import oracle as O

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build not present")

AIR = (287.05, 1.4)


def port(kind, first, second, cd=0.8, area=1e-4, conductance=1e-6, opening=1.0):
    return (kind, 0, first, second, cd, area, conductance, opening)


def random_case(n=4000, seed=11):
    rng = np.random.default_rng(seed)
    zones = [(p, t) for p, t in zip(rng.uniform(6e4, 3e5, 64), rng.uniform(250.0, 330.0, 64))]
    zones += [zones[0]]  # a zone at the same pressure as zone 0: equilibrium ports
    ports = []
    for k in range(n):
        a, b = rng.integers(0, len(zones), 2)
        if k % 50 == 0:
            a, b = 0, len(zones) - 1
        opening = 0.0 if k % 37 == 0 else rng.uniform(0.05, 1.0)
        kind = abi.PORT_CONDUCTANCE if k % 3 == 0 else abi.PORT_ORIFICE
        ports.append(port(kind, int(a), int(b), cd=rng.uniform(0.3, 1.0), area=rng.uniform(1e-6, 1e-2),
                          conductance=rng.uniform(1e-8, 1e-4), opening=opening))
    return zones, ports


def refusals():
    """(air, zones, ports, refusing port) per case the reference throws on."""
    good = [(101325.0, 293.15), (150000.0, 300.0)]
    ok = port(abi.PORT_ORIFICE, 0, 1)
    cases = []
    for bad in (port(abi.PORT_ORIFICE, 0, 1, opening=1.5), port(abi.PORT_ORIFICE, 0, 1, cd=0.0),
                port(abi.PORT_ORIFICE, 0, 1, cd=1.01), port(abi.PORT_ORIFICE, 0, 1, area=np.inf),
                port(abi.PORT_CONDUCTANCE, 0, 1, conductance=-1.0), port(abi.PORT_CONDUCTANCE, 0, 1, opening=np.nan),
                port(7, 0, 1), port(abi.PORT_ORIFICE, 0, 2), port(abi.PORT_CONDUCTANCE, 2, 1)):
        cases.append((AIR, good + [(np.nan, 300.0)], [ok, ok, bad, ok], 2))
    cases.append((AIR, good + [(1e5, -1.0)], [ok, port(abi.PORT_ORIFICE, 2, 0)], 1))
    cases.append(((287.05, 1.0), good, [port(abi.PORT_CONDUCTANCE, 0, 1), ok], 1))  # air checked by orifices only
    cases.append(((-1.0, 1.4), good, [ok], 0))
    cases.append((AIR, [(1e300, 300.0), (1.0, 300.0)], [ok, port(abi.PORT_CONDUCTANCE, 0, 1, conductance=1e10)], 1))
    return cases


@needs_ref
def test_reference_flow_laws_follow_their_closed_forms():
    """Pins the reference build: choked flow is Cd A p / sqrt(R T) times
    sqrt(gamma) (2 / (gamma + 1))^((gamma + 1) / (2 (gamma - 1))), the
    critical ratio (2 / (gamma + 1))^(gamma / (gamma - 1)), subsonic flow the
    isentropic nozzle law, and the conductance law G s (p1 - p2)."""
    zones = [(300000.0, 300.0), (101325.0, 290.0), (250000.0, 310.0)]
    ports = [port(abi.PORT_ORIFICE, 0, 1, cd=0.7, area=2e-4, opening=0.5),
             port(abi.PORT_ORIFICE, 0, 2, cd=0.9, area=1e-4),
             port(abi.PORT_CONDUCTANCE, 1, 2, conductance=3e-7, opening=0.25),
             port(abi.PORT_ORIFICE, 1, 1)]
    status, flows, failed = O.ref_port_mass_flows(zones, ports, AIR)
    assert status == 0 and failed == len(ports)
    R, g = AIR
    crit = (2 / (g + 1)) ** (g / (g - 1))
    assert crit == pytest.approx(0.528281787717174, rel=1e-14)
    choked = flows[0]
    assert choked["choked"] == 1 and choked["direction"] == abi.FLOW_FIRST_TO_SECOND
    assert choked["critical_pressure_ratio"] == pytest.approx(crit, rel=1e-15)
    expect = 0.7 * 2e-4 * 0.5 * 3e5 / np.sqrt(R * 300.0) * np.sqrt(g) * (2 / (g + 1)) ** ((g + 1) / (2 * (g - 1)))
    assert choked["magnitude"] == pytest.approx(expect, rel=1e-14)
    sub = flows[1]
    r = 250000.0 / 300000.0
    expect = 0.9 * 1e-4 * 3e5 / np.sqrt(R * 300.0) * np.sqrt(2 * g / (g - 1) * (r ** (2 / g) - r ** ((g + 1) / g)))
    assert sub["choked"] == 0 and sub["pressure_ratio"] == r and sub["magnitude"] == pytest.approx(expect, rel=1e-14)
    lin = flows[2]
    assert lin["signed_mass_rate"] == 3e-7 * 0.25 * (101325.0 - 250000.0)
    assert lin["direction"] == abi.FLOW_SECOND_TO_FIRST and lin["critical_pressure_ratio"] == 1.0
    assert flows[3]["direction"] == abi.FLOW_EQUILIBRIUM and flows[3]["magnitude"] == 0.0
    for air, z, p, k in refusals():
        status, _, failed = O.ref_port_mass_flows(z, p, air)
        if k is not None and max(max(q[2], q[3]) for q in p) < len(z):
            assert status == 1 and failed == k


@pytest.mark.gpu
@needs_ref
def test_device_port_flows_equal_the_reference(cuda_device):
    zones, ports = random_case()
    flows = sw.port_mass_flows(zones, ports, AIR)
    status, ref, failed = O.ref_port_mass_flows(zones, ports, AIR)
    assert status == 0 and failed == len(ports)
    kinds = np.array([p[0] for p in ports])
    lin, ori = kinds == abi.PORT_CONDUCTANCE, kinds == abi.PORT_ORIFICE
    assert flows[lin].tobytes() == ref[lin].tobytes()
    for f in ("direction", "choked"):
        np.testing.assert_array_equal(flows[ori][f], ref[ori][f])
    for f in ("signed_mass_rate", "magnitude", "pressure_ratio", "critical_pressure_ratio"):
        np.testing.assert_allclose(flows[ori][f], ref[ori][f], rtol=1e-12, atol=0.0)
    assert (flows[ori]["magnitude"] == ref[ori]["magnitude"]).mean() > 0.8  # 0.86 measured on B200
    # every regime occurs: choked, subsonic, equilibrium, closed
    assert flows["choked"].any() and (flows[ori]["choked"] == 0).any()
    assert (flows["direction"] == abi.FLOW_EQUILIBRIUM).sum() > len(ports) // 40


@pytest.mark.gpu
@needs_ref
def test_device_refuses_the_ports_the_reference_refuses(cuda_device):
    for air, zones, ports, k in refusals():
        status, _, failed = O.ref_port_mass_flows(zones, ports, air)
        if max(max(q[2], q[3]) for q in ports) >= len(zones):
            assert status == 2
            with pytest.raises(sw.OutOfRange):
                sw.port_mass_flows(zones, ports, air)
            continue
        assert status == 1 and failed == k
        with pytest.raises(sw.InvalidArgument) as e:
            sw.port_mass_flows(zones, ports, air)
        assert e.value.port == k
    assert len(sw.port_mass_flows([], [], AIR)) == 0


@pytest.mark.gpu
def test_device_array_port_flows_equal_the_host_form(cuda_device):
    """swb_port_mass_flows_device on device arrays (no allocation, no
    synchronisation) gives the host form's flows byte for byte, and reports
    the first refused port -- a zone index past the zone count included --
    through the device word."""
    import ctypes as C

    import torch

    zones, ports = random_case(n=3000, seed=5)
    z = np.array(zones, dtype=abi.ZONE_DTYPE)
    p = np.array(ports, dtype=abi.PORT_DTYPE)
    lib = abi.library()
    air = abi.AirProperties(*AIR)
    stream = torch.cuda.Stream()

    def device_flows(pp):
        dz = torch.from_numpy(z.view(np.uint8).copy()).cuda()
        dp = torch.from_numpy(pp.view(np.uint8).copy()).cuda()
        out = torch.zeros(len(pp) * abi.FLOW_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
        failed = torch.zeros(1, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        sw._check(lib.swb_port_mass_flows_device(C.byref(air), dz.data_ptr(), len(z), dp.data_ptr(), len(pp),
                                                 out.data_ptr(), failed.data_ptr(), C.c_void_p(stream.cuda_stream)))
        stream.synchronize()
        return out.cpu().numpy().view(abi.FLOW_DTYPE), int(failed.cpu().item())

    good = p[[k for k in range(len(p)) if p[k]["opening_fraction"] > 0.0]]
    flows, failed = device_flows(good)
    assert failed == len(good)
    assert flows.tobytes() == sw.port_mass_flows(z, good, AIR).tobytes()
    bad = good.copy()
    bad[100]["second"] = len(z) + 3  # unknown zone
    bad[700]["discharge_coefficient"] = 2.0  # refused constant
    _, failed = device_flows(bad)
    assert failed == 100
