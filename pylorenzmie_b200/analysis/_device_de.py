'''Differential evolution with the whole search on the GPU.

The reference's estimators (analysis/DEEstimator.py:158-166,
analysis/RadialEstimator.py:150-158) run scipy's differential_evolution
on the host; run_populations (``_de``) keeps scipy's exact algorithm and
random stream, so each generation still costs per-candidate host work.
``device_searches`` moves the search itself to the device: every
generation of every running search is three launches -- the trial
populations and their sphere records (lmb_de_trial), the Mie coefficients
and FP64 chi^2 of every trial against its own crop (lmb_sphere_ab,
lmb_chi2_crops), the selection and convergence test (lmb_de_select) --
with no host work between generations; the host reads the finished flags
every few generations and drops the finished searches from the launches.

The algorithm is scipy's best1bin with deferred updating, latin-hypercube
start, dithered mutation, binomial crossover and scipy's convergence test,
with the population energies in FP64 (the reference's model; no FP32
overflow to re-evaluate).  Its random numbers are a counter-based hash
(keyed by the search's seed), so a seeded search is reproducible but is
not the search scipy makes: estimates agree with scipy's in distribution,
not bit for bit.  The estimators select it with ``device_search=True``.
'''
import numpy as np
import torch
from scipy.optimize import OptimizeResult

from .. import _native
from .._device import ptr, stream_handle
from ..theory import _kernels as K
from ._de import _DEFAULTS, supported
from ._population import CropPopulations, _Candidates, SPHERE_KEYS

_CHECK_EVERY = 8       # generations between reads of the finished flags


def _key(seed, rng):
    '''64-bit key of a search's random stream.'''
    if seed is None:
        return int(rng.integers(0, 2 ** 63))
    if isinstance(seed, (np.random.RandomState, np.random.Generator)):
        return int(seed.randint(0, 2 ** 62) if isinstance(
            seed, np.random.RandomState) else seed.integers(0, 2 ** 62))
    return int(np.random.default_rng(int(seed)).integers(0, 2 ** 63))


def _lhs(rng, N, P):
    '''Latin-hypercube start in the unit cube, as scipy's.'''
    seg = 1.0 / N
    samples = (seg * rng.uniform(size=(N, P)) +
               np.linspace(0., 1., N, endpoint=False)[:, None])
    pop = np.zeros_like(samples)
    for j in range(P):
        pop[:, j] = samples[rng.permutation(N), j]
    return pop


def device_searches(searches):
    '''The searches (dicts of run_search's arguments) on the GPU, all in one
    generation loop.  They must share the device, instrument, noise,
    aberration, free variables, population size and mutation settings (the
    estimators' searches of a frame do) and be ones run_search would send
    to the GPU (batchable models, settings ``supported``).  Returns one
    OptimizeResult per search (x, fun, nit, nfev, success, message).'''
    first = searches[0]
    variables = list(first['variables'])
    P = len(variables)
    bounds = [np.array(sr['bounds'], dtype=float).T for sr in searches]
    S = len(searches)
    settings = dict(_DEFAULTS)
    settings.update(first['settings'] or {})
    for sr in searches:
        if list(sr['variables']) != variables or not supported(sr['settings']):
            raise ValueError('device searches share their variables and use '
                             'the estimators\' settings')
    fixed = [np.count_nonzero(b[0] == b[1]) for b in bounds]
    N = max(5, first['popsize'] * max(1, P - fixed[0]))
    if any(max(5, sr['popsize'] * max(1, P - f)) != N
           for sr, f in zip(searches, fixed)):
        raise ValueError('device searches share their population size')
    most = 65535 // N      # candidates per chi^2 launch
    if S > most:
        return (device_searches(searches[:most]) +
                device_searches(searches[most:]))
    mutation = settings['mutation']
    if hasattr(mutation, '__iter__') and len(mutation) > 1:
        mlo, mhi = sorted([float(mutation[0]), float(mutation[1])])
    else:
        mlo = mhi = float(mutation)
    pop_model = CropPopulations([(sr['model'], sr['data'], sr['coords'],
                                  variables) for sr in searches],
                                first['noise'])
    dev = pop_model.device
    lib = _native.load()
    glob = np.random.default_rng()
    keys, pops, mids, spans, bases = [], [], [], [], []
    tol, atol, maxiter, cr = [], [], [], []
    for sr, b in zip(searches, bounds):
        s = dict(_DEFAULTS)
        s.update(sr['settings'] or {})
        seed = sr['seed']
        keys.append(_key(seed, glob))
        start_rng = (np.random.default_rng(keys[-1]) if seed is not None
                     else glob)
        pops.append(_lhs(start_rng, N, P))
        mids.append(0.5 * (b[0] + b[1]))
        spans.append(np.fabs(b[0] - b[1]))
        bases.append(_Candidates(sr['model'], variables).base)
        tol.append(s['tol'])
        atol.append(s['atol'])
        maxiter.append(1000 if s['maxiter'] is None else int(s['maxiter']))
        cr.append(s['recombination'])

    def dt(a, dtype=torch.float64):
        return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype,
                               device=dev)
    d_pop = dt(np.array(pops))
    d_trial = torch.empty_like(d_pop)
    d_energy = torch.full((S, N), np.inf, dtype=torch.float64, device=dev)
    d_keys = torch.as_tensor(np.array(keys, dtype=np.uint64).view(np.int64),
                             device=dev)
    d_cr, d_mid, d_span = dt(cr), dt(np.array(mids)), dt(np.array(spans))
    d_base = dt(np.array(bases))
    d_slots = dt([SPHERE_KEYS.index(v) for v in variables], torch.int32)
    d_tol, d_atol = dt(tol), dt(atol)
    d_maxiter = dt(maxiter, torch.int32)
    d_nit = torch.zeros(S, dtype=torch.int32, device=dev)
    d_done = torch.zeros(S, dtype=torch.int32, device=dev)
    d_spheres = torch.empty((S * N, 6), dtype=torch.float64, device=dev)
    item_start = torch.arange(S * N + 1, dtype=torch.int32, device=dev)
    # the searches still running, by position: their candidates are
    # evaluated (sphere records and energies laid out by position)
    state = {}

    def set_live(live):
        state['L'] = len(live)
        state['live'] = torch.as_tensor(np.asarray(live, dtype=np.int32),
                                        device=dev)
        state['crop'] = state['live'].repeat_interleave(N)
    set_live(np.arange(S))
    # capacity: the largest sphere the bounds allow
    hi = np.array([b[1] for b in bounds])
    lo = np.array([b[0] for b in bounds])
    corner = np.array(bases)
    for j, v in enumerate(variables):
        corner[:, SPHERE_KEYS.index(v)] = np.maximum(hi[:, j], lo[:, j])
    cap = K.nmax_cap_for(corner[:, 3], corner[:, 4], corner[:, 5],
                         pop_model.n_m, pop_model.wavelength)
    stream = stream_handle(dev)

    def trial(generation, copy_only):
        _native.check(lib.lmb_de_trial(
            S, state['L'], ptr(state['live']), N, P, ptr(d_pop), ptr(d_trial),
            ptr(d_keys), generation, mlo, mhi, ptr(d_cr), ptr(d_mid),
            ptr(d_span), ptr(d_base), ptr(d_slots), ptr(d_done),
            int(copy_only), ptr(d_spheres), stream), 'lmb_de_trial')

    # the evaluation's buffers, made once: a generation allocates nothing
    M = S * N
    d_ab = torch.empty((M, cap + 1, 2, 2), dtype=torch.float64, device=dev)
    d_nmax = torch.empty(M, dtype=torch.int32, device=dev)
    d_status = torch.empty(M, dtype=torch.int32, device=dev)
    d_chi2 = torch.empty(M, dtype=torch.float64, device=dev)
    d_bad = torch.empty(M, dtype=torch.int32, device=dev)
    ws_bytes = lib.lmb_chi2_workspace_bytes(int(pop_model.max_npts), M)
    d_ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    coords, data = pop_model.coords.contiguous(), pop_model.data.contiguous()
    flags = K._flags(True, True, True)

    def energies():
        m = state['L'] * N
        _native.check(lib.lmb_sphere_ab(
            ptr(d_spheres), m, float(pop_model.n_m),
            float(pop_model.wavelength), cap, ptr(d_ab), None, ptr(d_nmax),
            ptr(d_status), stream), 'lmb_sphere_ab')
        _native.check(lib.lmb_chi2_crops(
            ptr(coords), coords.shape[1], ptr(data), float(pop_model.noise),
            ptr(pop_model.crop_start), S, ptr(state['crop']),
            int(pop_model.max_npts), ptr(d_spheres), ptr(item_start), m,
            ptr(d_ab), ptr(d_nmax), cap, float(pop_model.k), flags,
            ptr(d_chi2), ptr(d_bad), ptr(d_ws), ws_bytes, stream,
            float(pop_model.aberr)), 'lmb_chi2_crops')
        return d_chi2

    def select(e, first_call):
        _native.check(lib.lmb_de_select(
            S, state['L'], ptr(state['live']), N, P, ptr(d_pop),
            ptr(d_energy), ptr(d_trial), ptr(e), ptr(d_tol), ptr(d_atol),
            ptr(d_maxiter), ptr(d_nit), ptr(d_done), int(first_call),
            stream), 'lmb_de_select')

    trial(0, True)
    select(energies(), True)
    limit = int(max(maxiter))
    for generation in range(1, limit + 1):
        trial(generation, False)
        select(energies(), False)
        if generation % _CHECK_EVERY == 0 or generation == limit:
            live = np.flatnonzero(d_done.cpu().numpy() == 0)
            if not len(live):
                break
            if len(live) < state['L']:
                set_live(live)
    pop = d_pop.cpu().numpy()
    energy = d_energy.cpu().numpy()
    nit = d_nit.cpu().numpy()
    done = d_done.cpu().numpy()
    out = []
    for s in range(S):
        x = mids[s] + (pop[s, 0] - 0.5) * spans[s]
        ok = done[s] == 1
        out.append(OptimizeResult(
            x=x, fun=energy[s, 0], nit=int(nit[s]), nfev=int(nit[s]) + 1,
            success=bool(ok),
            message=('Optimization terminated successfully.' if ok else
                     'Maximum number of iterations has been exceeded.'),
            population=mids[s] + (pop[s] - 0.5) * spans[s],
            population_energies=energy[s]))
    return out
