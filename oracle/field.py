"""CPU oracle of the resolved-field tissue step: cells facing finite extracellular nodes.

TEST INFRASTRUCTURE ONLY, like oracle/tissue.py: only ``tests/`` and ``bench.py``'s CPU baseline
leg may import it, as the parity reference or the timed CPU baseline.

Restates, for one world at a time with dense node-space algebra (small worlds), the reference's
step of ``cells.model.resolved_pump_tissue@1`` under ``cells.solver.imex_ars222_face_
electromigration@1`` with the factored field solver (``capacitive_reduction_gauged_damped_
newton@2``):

* ``bind``: capacitor components by union of membranes, one representative per floating
  component (its lowest outside node), the floating basis and the face and junction incidences,
  the capacitor matrix and its scaled, reduced Cholesky factor (src/cells/numerics/
  surface_field.py:253-361, representative :237-250);
* ``capacitor_solve``, ``offset_solve`` (:596-611) and the gauged damped Newton on the floating
  offsets, with its backtracking and acceptance (``solve``, :614-855; the junction slope of
  numerics/tissue_field.py:186-190);
* ``transport`` with faces (numerics/surface_transport.py:298-386) and ``logmean``
  (numerics/extracellular_field.py:48-62);
* the readouts the step takes (models/surface_kinetic.py:221-410: the start potentials, the
  extracellular rate that predicts the operator time, the validity);
* ``explicit_rates``, ``implicit_rates``, ``face_weights``, ``drift_flux``, the face Laplacian,
  ``factor_operator`` and ``solve_operator`` (numerics/surface_imex.py:123-278), the electrode
  increment from ``capacitor_change`` (models/surface_tissue.py:350-395) and the ARS(2,2,2)
  ``imex_step`` (models/surface_pump.py:158-362), with ``domain_valid`` (surface_tissue.py:
  396-422).

Pinned against the reference's own step (tests/golden/make_golden.py, ``field_*.npz``).
State fields follow the reference's STATE_TYPE (src/cells/models/surface_kinetic.py:36-44)
without channels: cell arrays [S, N] or [N], outside-node arrays [S, O] or [O], junction arrays
[S, E] or [E], face arrays [S, F] or [F].
"""

from __future__ import annotations

from typing import NamedTuple

import numpy as np

from oracle import tissue as T
from oracle.n2 import cholesky_solve

F, R, K = T.F, T.R, T.CHARGE_PER_FMOL
MOL_PER_FMOL = T.MOL_PER_FMOL
Z = T.VALENCE[:, None]
CURRENT_ATOL_A = 1e-23  # surface_field.py:40
CURRENT_RTOL = 2e-12
NEWTON_TARGET = 0.01
MAX_ITERATIONS, MAX_BACKTRACKS = 16, 12


class FieldState(NamedTuple):
    amount_increment: np.ndarray
    extracellular_increment: np.ndarray
    membrane_transferred: np.ndarray
    junction_transferred: np.ndarray
    face_transferred: np.ndarray
    reservoir_supplied: np.ndarray
    membrane_dissipated: np.ndarray
    junction_dissipated: np.ndarray
    face_dissipated: np.ndarray
    electrode_charge: np.ndarray
    reservoir_work: np.ndarray
    electrode_work: np.ndarray
    junction_gate: np.ndarray
    pump_cycles: np.ndarray
    pump_dissipated: np.ndarray
    metabolic_work: np.ndarray


class Control(NamedTuple):
    membrane: np.ndarray  # [N]
    junction: np.ndarray  # [E]
    pump: np.ndarray  # [N]


class Topo(NamedTuple):
    n: int
    o: int
    capacitor: np.ndarray  # [size, size]
    scale: float
    factor: np.ndarray  # lower factor of the capacitor solve matrix
    fixed: np.ndarray  # [size] bool
    basis: np.ndarray  # [size, K]
    face_incidence: np.ndarray  # [K, F]
    junction_incidence: np.ndarray  # [K, E]
    required: np.ndarray  # [size] bool: active and not held
    free: np.ndarray  # [size] bool: the operator's solved nodes
    held: np.ndarray  # [size] the clamps' potentials


def initial_state(w):
    n, o, e, f = w.cells, w.nodes, w.edges, w.faces
    return FieldState(
        np.zeros((3, n)), np.zeros((3, o)), np.zeros((3, n)), np.zeros((3, e)),
        np.zeros((3, f)), np.zeros((3, o)), np.zeros(n), np.zeros(e), np.zeros(f),
        np.zeros(o), np.zeros(o), np.zeros(o), np.asarray(w.gate_initial, dtype=float).copy(),
        np.zeros(n), np.zeros(n), np.zeros(n),
    )  # fmt: skip


def full_control(w):
    return Control(np.ones(w.cells), np.ones(w.edges), np.ones(w.cells))


SPARSE_ABOVE = 3000  # node-space size above which bind(w) takes the sparse containers


def bind(w, sparse=None):
    """surface_field.bind (:253-361) for a world with no gauge and every node active.

    sparse (default: node space above SPARSE_ABOVE): the same algebra in scipy.sparse containers
    with sparse LU solves (``_bind_sparse``), for grids whose dense node-space matrices do not fit
    (the 128x128 benchmark grid: 17,408 nodes, 16,4xx floating offsets). Dense is the branch
    pinned bit for bit to the reference; sparse agrees with it to rounding (tests)."""
    if sparse is None:
        sparse = w.cells + w.nodes > SPARSE_ABOVE
    if sparse:
        return _bind_sparse(w)
    n, o = w.cells, w.nodes
    size = n + o
    parent = list(range(size))

    def root(i):
        while parent[i] != i:
            i = parent[i]
        return i

    capacitor = np.zeros((size, size))
    for k in range(n):  # membrane k is cell k's patch
        i, j = k, n + int(w.cell_node[k])
        c = w.capacitance[k]
        parent[root(j)] = root(i)
        capacitor[i, i] += c
        capacitor[j, j] += c
        capacitor[i, j] -= c
        capacitor[j, i] -= c
    groups = {}
    for i in range(size):
        groups.setdefault(root(i), []).append(i)
    reservoirs = set((n + np.flatnonzero(w.reservoir)).tolist())
    fixed = np.zeros(size, dtype=bool)
    fixed[list(reservoirs)] = True
    floating = []
    for members in groups.values():
        if reservoirs.intersection(members):
            continue
        chosen = min(i for i in members if i >= n)
        fixed[chosen] = True
        floating.append(np.isin(np.arange(size), members).astype(float))
    basis = np.asarray(floating).reshape((-1, size)).T
    scale = np.max(np.abs(capacitor))
    solve_matrix = np.where((~fixed)[:, None] & (~fixed)[None, :], capacitor / scale, 0.0)
    solve_matrix += np.diag(fixed.astype(float))
    factor = np.linalg.cholesky(solve_matrix)
    held_out = np.asarray(w.reservoir, dtype=bool)
    clamp = np.r_[np.zeros(n, dtype=bool), held_out]
    return Topo(
        n, o, capacitor, scale, factor, fixed, basis,
        (basis[n + w.face_sender] - basis[n + w.face_receiver]).T,
        (basis[w.sender] - basis[w.receiver]).T,
        ~np.r_[np.zeros(n, dtype=bool), held_out], ~clamp,
        np.where(clamp, np.r_[np.zeros(n), w.boundary_V], 0.0),
    )  # fmt: skip


def _bind_sparse(w):
    """bind's reduction with scipy.sparse containers: the same components (a cell joins its
    node's; each other node is its own), representatives, clamps and scaled capacitor matrix; the
    basis and incidences as sparse matrices; the scaled reduced capacitor matrix factored by a
    sparse LU (SuperLU) instead of a dense Cholesky."""
    import scipy.sparse as sp

    n, o = w.cells, w.nodes
    size = n + o
    parent = list(range(size))

    def root(i):
        while parent[i] != i:
            i = parent[i]
        return i

    rows, cols, vals = [], [], []
    for k in range(n):
        i, j = k, n + int(w.cell_node[k])
        c = w.capacitance[k]
        parent[root(j)] = root(i)
        rows += [i, j, i, j]
        cols += [i, j, j, i]
        vals += [c, c, -c, -c]
    capacitor = sp.csr_matrix((vals, (rows, cols)), shape=(size, size))
    groups = {}
    for i in range(size):
        groups.setdefault(root(i), []).append(i)
    reservoirs = set((n + np.flatnonzero(w.reservoir)).tolist())
    fixed = np.zeros(size, dtype=bool)
    fixed[list(reservoirs)] = True
    brow, bcol, k_count = [], [], 0
    for members in groups.values():
        if reservoirs.intersection(members):
            continue
        chosen = min(i for i in members if i >= n)
        fixed[chosen] = True
        brow += members
        bcol += [k_count] * len(members)
        k_count += 1
    basis = sp.csr_matrix((np.ones(len(brow)), (brow, bcol)), shape=(size, k_count))
    scale = float(np.max(np.abs(capacitor.data)))
    free = sp.diags((~fixed).astype(float))
    solve_matrix = (free @ (capacitor / scale) @ free + sp.diags(fixed.astype(float))).tocsc()
    factor = _SparseFactor(solve_matrix)
    held_out = np.asarray(w.reservoir, dtype=bool)
    clamp = np.r_[np.zeros(n, dtype=bool), held_out]
    return Topo(
        n, o, capacitor, scale, factor, fixed, basis,
        (basis[n + w.face_sender] - basis[n + w.face_receiver]).T.tocsr(),
        (basis[w.sender] - basis[w.receiver]).T.tocsr(),
        ~np.r_[np.zeros(n, dtype=bool), held_out], ~clamp,
        np.where(clamp, np.r_[np.zeros(n), w.boundary_V], 0.0),
    )  # fmt: skip


class _SparseFactor:
    """A sparse LU of a symmetric positive definite matrix, standing in for its dense Cholesky
    factor in the sparse branch (``solve`` in place of cholesky_solve)."""

    def __init__(self, matrix):
        from scipy.sparse.linalg import splu

        self.lu = splu(matrix.tocsc())
        diag = self.lu.U.diagonal()
        self.valid = bool(np.all(np.isfinite(diag)) and np.all(diag > 0))

    def solve(self, rhs):
        return self.lu.solve(np.asarray(rhs, dtype=float))


def _is_sparse(m):
    return hasattr(m, "tocsr")


def _factor_solve(factor, rhs):
    return factor.solve(rhs) if isinstance(factor, _SparseFactor) else cholesky_solve(factor, rhs)


def capacitor_solve(charge, boundary, tp):
    """_capacitor_solve (surface_field.py:596-600) with the factored layout's solve."""
    rhs = np.where(~tp.fixed, (charge - tp.capacitor @ boundary) / tp.scale, 0.0)
    return _factor_solve(tp.factor, rhs) + boundary


def offset_solve(matrix, rhs):
    """_offset_solve (:603-611): every offset free (no gauge)."""
    if rhs.size == 0:
        return np.zeros_like(rhs)
    if _is_sparse(matrix):
        from scipy.sparse.linalg import spsolve

        scale = float(np.max(np.abs(matrix.data), initial=0.0)) or 1.0
        return spsolve((matrix / scale).tocsc(), rhs / scale)
    scale = np.max(np.abs(matrix), initial=0.0)
    scale = np.where(scale > 0, scale, 1.0)
    return np.linalg.solve(matrix / scale, rhs / scale)


def _weighted_gram(incidence, weight):
    """incidence diag(weight) incidence^T, dense or sparse."""
    if _is_sparse(incidence):
        import scipy.sparse as sp

        return (incidence @ sp.diags(weight) @ incidence.T).tocsr()
    return (incidence * weight) @ incidence.T


def logmean(left, right):
    """extracellular_field.logmean (:48-62)."""
    middle = 0.5 * left + 0.5 * right
    difference = left - right
    ratio = (0.5 * difference) / middle
    near = np.abs(ratio) < 0.5
    with np.errstate(all="ignore"):
        log = np.where(near, 2 * np.arctanh(np.where(near, ratio, 0.0)),
                       np.log(left) - np.log(right))
        small = np.abs(ratio) < 1e-4
        square = ratio * ratio
        mean = np.where(small, middle * (1 - square / 3 - 4 * square * square / 45),
                        difference / np.where(small, 1.0, log))
    return mean, log


def _sum(values, owners, size):
    out = np.zeros((*values.shape[:-1], size))
    np.add.at(out, (Ellipsis, owners), values)
    return out


class Transport(NamedTuple):
    cell: np.ndarray
    outside: np.ndarray
    supply: np.ndarray
    membrane_dv: np.ndarray
    membrane_flux: np.ndarray
    membrane_mu: np.ndarray
    membrane_current: np.ndarray
    membrane_dissipation: np.ndarray
    junction_dv: np.ndarray
    junction_flux: np.ndarray
    junction_mu: np.ndarray
    junction_current: np.ndarray
    junction_dissipation: np.ndarray
    face_dv: np.ndarray
    face_flux: np.ndarray
    face_mu: np.ndarray
    face_current: np.ndarray
    face_dissipation: np.ndarray
    valid: bool


def transport(ci, co, phi_cell, phi_out, membrane_open, junction_open, w):
    """surface_transport.transport (:298-386)."""
    n, o = w.cells, w.nodes
    valid = (np.all(np.isfinite(ci) & (ci > 0)) & np.all(np.isfinite(co) & (co > 0))
             & np.all(np.isfinite(phi_cell)) & np.all(np.isfinite(phi_out)))  # fmt: skip
    for control in (membrane_open, junction_open):
        valid = valid & np.all(np.isfinite(control) & (control >= 0) & (control <= 1))
    rt = R * w.temperature
    routes = (
        ("membrane", ci, co[:, w.cell_node], phi_cell - phi_out[w.cell_node], membrane_open),
        ("junction", ci[:, w.sender], ci[:, w.receiver], phi_cell[w.sender] - phi_cell[w.receiver],
         junction_open),
        ("face", co[:, w.face_sender], co[:, w.face_receiver],
         phi_out[w.face_sender] - phi_out[w.face_receiver], None),
    )  # fmt: skip
    values = []
    with np.errstate(all="ignore"):
        for prefix, left, right, dv, opening in routes:
            mu = rt * (np.log(left) - np.log(right)) + Z * F * dv
            if prefix == "face":
                mean, _ = logmean(left, right)
                flux = w.face_factor * mean * mu / (rt * MOL_PER_FMOL)
            elif prefix == "membrane":
                flux = T.route_flux(left, right, dv, w.temperature, w.area, w.permeability, opening)
            else:
                flux = T.route_flux(left, right, dv, w.temperature, w.junction_area,
                                    w.junction_permeability, opening)
            current = K * np.sum(Z * flux, axis=0)
            dissipation = 1e-3 * np.sum(flux * mu, axis=0)
            values.append((dv, flux, mu, current, dissipation))
            valid = valid & np.all(np.abs(Z * F * dv / rt) <= T.MAX_ABS_X)
            valid = valid & np.all(np.isfinite(flux)) & np.all(np.isfinite(dissipation))
    membrane, junction, face = (v[1] for v in values)
    cell = -_sum(membrane, np.arange(n), n)
    cell += _sum(-junction, w.sender, n)
    cell += _sum(junction, w.receiver, n)
    outside = _sum(membrane, w.cell_node, o)
    outside += _sum(-face, w.face_sender, o)
    outside += _sum(face, w.face_receiver, o)
    supply = np.where(w.reservoir, -outside, 0.0)
    finite = np.where(w.reservoir, 0.0, outside)
    flat = (cell, finite, supply, *(v for route in values for v in route))
    for value in flat:
        valid = valid & np.all(np.isfinite(value))
    return Transport(*flat, bool(valid))


def bernoulli_derivative(x):
    """numerics/tissue_field._bernoulli_derivative (:186-190)."""
    small = np.abs(x) < 1e-4
    a, b = np.where(small, x, 0.0), np.where(small, 1.0, x)
    with np.errstate(all="ignore"):
        em1 = np.expm1(b)
        return np.where(small, -0.5 + a / 6 - a**3 / 180, (em1 - b * np.exp(b)) / (em1 * em1))


class Field(NamedTuple):
    potential: np.ndarray  # [n + o]
    rates: Transport
    iterations: int
    converged: bool


def field_solve(ci, co, q_cell, q_out, membrane_open, junction_open, w, tp):
    """surface_field.solve (:614-855) for the factored layout, no forms faces."""
    n = w.cells
    charge = np.concatenate((q_cell, q_out))
    clamps = np.asarray(w.reservoir, dtype=bool)
    boundary = np.concatenate((np.zeros(n), np.where(clamps, w.boundary_V, 0.0)))
    base = capacitor_solve(charge, boundary, tp)
    domain = (np.all(np.isfinite(charge)) & np.all(np.isfinite(w.boundary_V))
              & np.all(np.where(clamps, True, w.boundary_V == 0)))  # fmt: skip
    rt = R * w.temperature
    mean, log = logmean(co[:, w.face_sender], co[:, w.face_receiver])
    weight = w.face_factor * mean
    conductance = F**2 / rt * np.sum(Z * Z * weight, axis=0)
    dv = base[n + w.face_sender] - base[n + w.face_receiver]
    face0 = F * np.sum(Z * weight * log, axis=0) + conductance * dv
    fi, ji = tp.face_incidence, tp.junction_incidence
    matrix = _weighted_gram(fi, conductance)
    initial_offset = offset_solve(matrix, -fi @ face0)

    def evaluate(offset):
        phi = base + tp.basis @ offset
        rates = transport(ci, co, phi[:n], phi[n:], membrane_open, junction_open, w)
        residual = fi @ rates.face_current + ji @ rates.junction_current
        scale = np.maximum(np.max(np.abs(rates.face_current), initial=0.0),
                           np.max(np.abs(rates.junction_current), initial=0.0))
        norm = np.max(np.abs(residual), initial=0.0) / (CURRENT_ATOL_A + CURRENT_RTOL * scale)
        x = Z * F * rates.junction_dv / rt
        a, b = ci[:, w.sender], ci[:, w.receiver]
        slope = (F**2 / rt * w.junction_area * junction_open
                 * np.sum(Z * Z * w.junction_permeability
                          * (-a * bernoulli_derivative(-x) - b * bernoulli_derivative(x)), axis=0))
        valid = (domain & rates.valid & np.isfinite(norm) & np.all(np.isfinite(phi))
                 & np.all(np.isfinite(slope) & (slope >= 0)))  # fmt: skip
        return phi, rates, residual, norm, slope, bool(valid)

    def iteration(count, offset):
        _, _, residual, norm, slope, _ = evaluate(offset)
        jac = matrix + _weighted_gram(ji, slope)
        delta = offset_solve(jac, -residual)
        before = np.max(np.abs(residual), initial=0.0)
        step, proposal, accepted = 0, offset, False
        while step < MAX_BACKTRACKS and not accepted:
            proposal = offset + delta * (0.5**step)
            _, _, r, norm, _, valid = evaluate(proposal)
            accepted = valid and (np.max(np.abs(r), initial=0.0) < before or norm <= NEWTON_TARGET)
            step += 1
        return count + 1, (proposal if accepted else offset), norm, accepted

    _, _, _, norm, _, valid = evaluate(initial_offset)
    count, offset, accepted = 0, initial_offset, valid
    while count < MAX_ITERATIONS and norm > NEWTON_TARGET and accepted:
        count, offset, norm, accepted = iteration(count, offset)
    phi, rates, _, norm, _, valid = evaluate(offset)
    rooted = accepted and norm <= NEWTON_TARGET
    cap_charge = tp.capacitor @ phi
    residual = np.where(tp.required, cap_charge - charge, 0.0)
    bound = T.CHARGE_ATOL_C + T.CHARGE_RTOL * np.maximum(np.abs(charge), np.abs(cap_charge))
    solved = tp.required & ~tp.fixed
    solved_norm = np.max(np.where(solved, np.abs(residual), 0.0) / bound)
    converged = bool(valid and rooted and solved_norm <= 1.0 and np.all(np.isfinite(phi)))
    return Field(phi, rates, count, converged)


def amounts(state, w):
    ci = (w.amount + state.amount_increment) / w.volume
    co = (w.outside_amount + state.extracellular_increment) / w.outside_volume
    return ci, co


def node_charge(state, w):
    """surface_pump.node_charge: initial charges plus z F dn (surface_tissue.charge_increment)."""
    return (w.initial_charge + K * np.sum(Z * state.amount_increment, axis=0),
            w.outside_charge + K * np.sum(Z * state.extracellular_increment, axis=0))


def _pump(ci, co, mu, w, availability):
    pump = w.pump
    args = (ci[0], co[1, w.cell_node], mu[0], mu[1], w.temperature, pump, w.pump_capacity,
            availability)
    cycles, energy, drive = T.pump_kinetics(*args)
    return cycles, energy, drive, T.pump_domain(*args)


def readouts(state, control, w, tp):
    """(start potentials, extracellular rate, valid) of surface_kinetic.readouts (:221-410)."""
    ci, co = amounts(state, w)
    qc, qo = node_charge(state, w)
    opening = control.junction * state.junction_gate
    fld = field_solve(ci, co, qc, qo, control.membrane, opening, w, tp)
    r = fld.rates
    cycles, _, _, pump_ok = _pump(ci, co, r.membrane_mu, w, control.pump)
    extra = -T.STOICHIOMETRY[:, None] * cycles
    out_extra = _sum(extra, w.cell_node, w.nodes)
    outside = r.outside + np.where(w.reservoir, 0.0, out_extra)
    gate_ok = T.gate_domain(state.junction_gate, r.junction_dv, w.gate_threshold, w.gate_minimum,
                            control.junction)
    valid = fld.converged and bool(np.all(pump_ok)) and bool(np.all(gate_ok))
    for value in control:
        valid = valid and bool(np.all(np.isfinite(value) & (value >= 0) & (value <= 1)))
    valid = valid and bool(np.all(np.isfinite(outside))) and domain_valid(state, w)
    return fld.potential, outside, valid


def face_weights(co, w):
    """surface_imex.face_weights (:123-134)."""
    left, right = co[:, w.face_sender], co[:, w.face_receiver]
    mean, _ = logmean(left, right)
    return w.face_factor * mean / MOL_PER_FMOL, np.log(left) - np.log(right)


def explicit_rates(state, potential, control, w):
    """surface_pump.explicit_rates (:158-240): every rate but the face drift."""
    n, o = w.cells, w.nodes
    ci, co = amounts(state, w)
    r = transport(ci, co, potential[:n], potential[n:], control.membrane,
                  control.junction * state.junction_gate, w)
    weight, log = face_weights(co, w)
    diffusion = weight * log
    cycles, energy, drive, pump_ok = _pump(ci, co, r.membrane_mu, w, control.pump)
    extra = -T.STOICHIOMETRY[:, None] * cycles
    inflow = (_sum(r.membrane_flux + extra, w.cell_node, o) - _sum(diffusion, w.face_sender, o)
              + _sum(diffusion, w.face_receiver, o))
    gate = T.gate_rhs(state.junction_gate, r.junction_dv, w.gate_threshold, w.gate_minimum)
    zo = np.zeros(o)
    rates = FieldState(
        r.cell - _sum(extra, np.arange(n), n),
        np.where(w.reservoir, 0.0, inflow),
        r.membrane_flux, r.junction_flux, diffusion,
        np.where(w.reservoir, -inflow, 0.0),
        r.membrane_dissipation, r.junction_dissipation, np.zeros(w.faces), zo, zo, zo,
        gate, cycles, -1e-3 * cycles * energy, -1e-3 * cycles * drive,
    )  # fmt: skip
    valid = r.valid and bool(np.all(pump_ok))
    valid = valid and bool(np.all(T.gate_domain(state.junction_gate, r.junction_dv,
                                                w.gate_threshold, w.gate_minimum,
                                                control.junction)))
    for value in (*control, *rates):
        valid = valid and bool(np.all(np.isfinite(value)))
    for value in control:
        valid = valid and bool(np.all((value >= 0) & (value <= 1)))
    return rates, valid


def implicit_rates(weight, potential, state, w):
    """surface_pump.implicit_rates (:243-256) with drift_flux (surface_imex.py:137-141)."""
    n, o = w.cells, w.nodes
    phi = potential[n:]
    dv = phi[w.face_sender] - phi[w.face_receiver]
    flux = weight * (Z * F / (R * w.temperature)) * dv
    inflow = _sum(flux, w.face_receiver, o) - _sum(flux, w.face_sender, o)
    zero = FieldState(*(np.zeros_like(v) for v in state))
    return zero._replace(extracellular_increment=np.where(w.reservoir, 0.0, inflow),
                         face_transferred=flux,
                         reservoir_supplied=np.where(w.reservoir, -inflow, 0.0))


def face_laplacian(weight, w, tp):
    """surface_imex.face_laplacian (:144-156), dense in the node space (sparse for a sparse
    bind)."""
    n = w.cells
    conductance = K * F / (R * w.temperature) * np.sum(Z**2 * weight, axis=0)
    a, b = n + w.face_sender, n + w.face_receiver
    size = tp.n + tp.o
    if _is_sparse(tp.capacitor):
        import scipy.sparse as sp

        rows = np.concatenate((a, b, a, b))
        cols = np.concatenate((a, b, b, a))
        vals = np.concatenate((conductance, conductance, -conductance, -conductance))
        return sp.csr_matrix((vals, (rows, cols)), shape=(size, size))
    parts = []
    for rows, cols in ((a, a), (b, b), (a, b), (b, a)):
        m = np.zeros((size, size))
        np.add.at(m, (rows, cols), conductance)
        parts.append(m)
    return parts[0] + parts[1] - parts[2] - parts[3]


class Operator(NamedTuple):
    factor: np.ndarray
    scale: np.ndarray
    matrix: np.ndarray
    held: np.ndarray
    free: np.ndarray


def factor_operator(coefficient, laplacian, tp):
    """surface_imex.factor_operator (:207-225), dense (sparse LU for a sparse bind)."""
    free = tp.free
    matrix = tp.capacitor + coefficient * laplacian
    if _is_sparse(matrix):
        import scipy.sparse as sp

        matrix = matrix.tocsr()
        diagonal = np.where(free, matrix.diagonal(), 1.0)
        scale = 1.0 / np.sqrt(np.where(diagonal > 0, diagonal, 1.0))
        keep = sp.diags(free.astype(float) * scale)
        reduced = (keep @ matrix @ keep + sp.diags((~free).astype(float))).tocsc()
        factor = _SparseFactor(reduced)
        valid = bool(np.all(diagonal > 0) and factor.valid)
        return Operator(factor, scale, matrix, tp.held, free), valid
    diagonal = np.where(free, np.diagonal(matrix), 1.0)
    scale = 1.0 / np.sqrt(np.where(diagonal > 0, diagonal, 1.0))
    reduced = np.where(free[:, None] & free[None, :], matrix * scale[:, None] * scale[None, :], 0.0)
    reduced += np.diag((~free).astype(float))
    factor = np.linalg.cholesky(reduced)
    valid = bool(np.all(diagonal > 0) and np.all(np.isfinite(factor)))
    return Operator(factor, scale, matrix, tp.held, free), valid


def solve_operator(charge, op):
    """surface_imex.solve_operator (:269-278), dense."""
    rhs = np.where(op.free, (charge - op.matrix @ op.held) * op.scale, 0.0)
    phi = np.where(op.free, _factor_solve(op.factor, rhs) * op.scale, op.held)
    return phi, np.where(op.free, op.matrix @ phi - charge, 0.0)


def _species_sum(amount):
    total = T.VALENCE[0] * amount[0]
    for s in range(1, amount.shape[0]):
        total = total + T.VALENCE[s] * amount[s]
    return total


def plate_charge(state, tp):
    """capacitor_change's plate charges (surface_tissue.py:358-395): C times the charge-only
    potentials of the increments."""
    q = K * np.concatenate((_species_sum(state.amount_increment),
                            _species_sum(state.extracellular_increment)))
    dp = capacitor_solve(q, np.zeros_like(q), tp)
    return tp.capacitor @ dp


def domain_valid(state, w):
    """surface_tissue.domain_valid (:396-422) with every slot active."""
    res = np.asarray(w.reservoir, dtype=bool)
    masks = (True, ~res, True, True, True, res, True, True, True, res, res, res)
    for v, mask in zip(state[:12], masks, strict=True):
        if not (np.all(np.isfinite(v)) and np.all(np.where(mask, True, v == 0))):
            return False
    ci = w.amount + state.amount_increment
    co = w.outside_amount + state.extracellular_increment
    if not (np.all(np.isfinite(ci) & (ci > 0)) and np.all(np.isfinite(co) & (co > 0))):
        return False
    for v, coefficient in ((state.membrane_transferred, w.permeability),
                           (state.junction_transferred, w.junction_permeability),
                           (state.face_transferred, w.face_factor)):
        if not np.all(np.where(coefficient > 0, True, v == 0)):
            return False
    return True


def _combine(state, dt, terms):
    result = state
    for weight, rates in terms:
        result = FieldState(*(y + (weight * dt) * d for y, d in zip(result, rates, strict=True)))
    return result


def imex_step(state, dt, control, w, tp):
    """surface_pump.imex_step (:259-362), ARS(2,2,2), operator time 1/2. (state, valid)."""
    n = w.cells
    e_mat = np.array([[0.0, 0.0, 0.0], [T.GAMMA, 0.0, 0.0], [T.DELTA, 1.0 - T.DELTA, 0.0]])
    i_mat = np.array([[0.0, 0.0, 0.0], [0.0, T.GAMMA, 0.0], [0.0, 1.0 - T.GAMMA, T.GAMMA]])
    start, outside_rate, valid = readouts(state, control, w, tp)
    amount = w.outside_amount + state.extracellular_increment
    predicted = amount + 0.5 * dt * outside_rate
    predicted = predicted / w.outside_volume
    valid = valid and bool(np.all(np.isfinite(predicted) & (predicted > 0)))
    weight, _ = face_weights(np.where(predicted > 0, predicted, 1.0), w)
    op, ok = factor_operator(i_mat[-1, -1] * dt, face_laplacian(weight, w, tp), tp)
    valid = valid and ok
    rates, ok = explicit_rates(state, start, control, w)
    explicit, implicit, valid = [rates], [None], valid and ok
    stage = state
    for i in range(1, 3):
        known = _combine(state, dt, [(e_mat[i, j], explicit[j]) for j in range(i)]
                         + [(i_mat[i, j], implicit[j]) for j in range(1, i)])
        qc, qo = node_charge(known, w)
        charge = np.concatenate((qc, qo))
        potential, residual = solve_operator(charge, op)
        scale = np.maximum(np.abs(charge), np.abs(op.matrix @ potential))
        valid = valid and bool(np.all(np.isfinite(potential)))
        valid = valid and bool(np.all(np.abs(residual) <= T.CHARGE_ATOL_C
                                      + T.CHARGE_RTOL * scale))
        drift = implicit_rates(weight, potential, state, w)
        implicit.append(drift)
        stage = _combine(known, dt, [(i_mat[i, i], drift)])
        if i < 2:
            rates, ok = explicit_rates(stage, potential, control, w)
            explicit.append(rates)
            valid = valid and ok

    def applied(name):
        return (sum(e_mat[2, j] * getattr(explicit[j], name) for j in range(2))
                + sum(i_mat[2, j] * getattr(implicit[j], name) for j in range(1, 3)))

    flux = applied("face_transferred")
    with np.errstate(all="ignore"):
        heat = 1e-3 * R * w.temperature * np.sum(
            np.where(weight > 0, flux * flux / np.where(weight > 0, weight, 1.0), 0.0), axis=0)
    start_plate, end_plate = plate_charge(state, tp), plate_charge(stage, tp)
    electrode = np.where(w.reservoir, end_plate[n:] - start_plate[n:], 0.0)
    co0 = w.outside_amount / w.outside_volume
    mu = R * w.temperature * np.log(co0) + Z * F * w.boundary_V
    stage = stage._replace(
        face_dissipated=state.face_dissipated + dt * heat,
        electrode_charge=state.electrode_charge + electrode,
        reservoir_work=state.reservoir_work
        + 1e-3 * np.sum(mu * (dt * applied("reservoir_supplied")), axis=0),
        electrode_work=state.electrode_work + 1e12 * w.boundary_V * electrode,
    )
    valid = valid and domain_valid(stage, w)
    for value in stage:
        valid = valid and bool(np.all(np.isfinite(value)))
    return (stage if valid else state), valid
