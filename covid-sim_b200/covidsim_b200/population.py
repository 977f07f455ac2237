"""Synthetic populations in the layout of cs_population.

Restates the steps of the reference's set-up (src/SetupModel.cpp) that shape the
hot path's inputs, vectorised with numpy:
  - microcell populations: multinomial over lognormal microcell densities (the
    reference's sequential binomial allocation, SetupModel.cpp:1137-1148, draws the
    same distribution);
  - households: sizes drawn from the household size distribution and truncated at
    microcell boundaries, people numbered microcell by microcell
    (SetupModel.cpp:1224-1253);
  - household locations uniform within their microcell;
  - ages drawn from a 17-band age distribution (capped at 84 as the reference does,
    SetupModel.cpp:1111), without the reference's household-composition rules;
  - places of four types with attendance by age band, located in microcells drawn
    in proportion to population, attendees assigned along a Z-order curve in runs of
    the place's size so that people attend nearby places (a stand-in for the
    reference's nearest-place kernel assignment, SetupModel.cpp:1989-2466), and
    each place split into groups of about PlaceTypeGroupSizeParam1 members.
"""
import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import abi
from .geometry import morton2

HH_SIZE_DIST = [0.28, 0.34, 0.16, 0.14, 0.05, 0.03]
# ages: roughly uniform to 60, then declining (17 five-year bands)
AGE_DIST = [1.0] * 12 + [0.9, 0.75, 0.55, 0.35, 0.25]

# attendance by age band per place type: (min, max, proportion) x 3 bands
# (primary, secondary, university, workplace), as in the reference's admin files
PLACE_AGE_BANDS = [
    [(5, 11, 0.928), (3, 5, 0.562), (21, 65, 0.0075)],
    [(11, 16, 0.974), (16, 18, 0.917), (21, 65, 0.0052)],
    [(18, 65, 0.0), (18, 21, 0.660), (21, 65, 0.0667)],
    [(16, 18, 0.340), (18, 21, 0.083), (21, 65, 0.883)],
]
PLACE_MEAN_SIZE = [230.0, 1000.0, 3300.0, 15.0]
GROUP_SIZE_PARAM1 = [25, 25, 100, 10]
WORKPLACE_POWER, WORKPLACE_OFFSET, WORKPLACE_MAX = 1.34, 5.35, 5000.0


@dataclass
class Population:
    n_people: int
    grid: dict
    person_hh: np.ndarray
    person_mcell: np.ndarray
    person_age: np.ndarray
    person_flags: np.ndarray
    person_place: np.ndarray      # [NPT, N]
    person_group: np.ndarray      # [NPT, N]
    hh_first: np.ndarray
    hh_nh: np.ndarray
    hh_nhr: np.ndarray
    hh_x: np.ndarray
    hh_y: np.ndarray
    mcell_cell: np.ndarray
    mcell_adunit: np.ndarray
    mcell_grid: np.ndarray        # microcell grid index of each populated microcell
    cell_grid: np.ndarray
    cell_start: np.ndarray
    cell_members: np.ndarray
    places: list = field(default_factory=list)  # per type: dict of arrays
    n_adunits: int = 1
    setup_info: dict = None       # set-up on the device: timings and counts

    @property
    def n_households(self):
        return len(self.hh_first)

    @property
    def n_cells(self):
        return len(self.cell_grid)

    @property
    def n_mcells(self):
        return len(self.mcell_cell)

    @property
    def num_place_types(self):
        return len(self.places)

    def to_c(self, lookup, hires):
        """cs_population pointing at this object's arrays (keep `self` alive)."""
        s = abi.cs_population()
        s.n_people, s.n_households, s.n_cells, s.n_mcells = self.n_people, self.n_households, self.n_cells, self.n_mcells
        s.num_place_types, s.n_adunits = self.num_place_types, self.n_adunits
        keep = []

        def ptr(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
            return a.ctypes.data

        s.person_hh = ptr(self.person_hh, np.int32)
        s.person_mcell = ptr(self.person_mcell, np.int32)
        s.person_age = ptr(self.person_age, np.uint8)
        s.person_flags = ptr(self.person_flags, np.uint8)
        s.person_place = ptr(self.person_place, np.int32)
        s.person_group = ptr(self.person_group, np.uint16)
        s.hh_first = ptr(self.hh_first, np.int32)
        s.hh_nh = ptr(self.hh_nh, np.uint16)
        s.hh_nhr = ptr(self.hh_nhr, np.uint16)
        s.hh_x = ptr(self.hh_x, np.float32)
        s.hh_y = ptr(self.hh_y, np.float32)
        s.mcell_cell = ptr(self.mcell_cell, np.int32)
        s.mcell_adunit = ptr(self.mcell_adunit, np.int32)
        s.cell_grid = ptr(self.cell_grid, np.int32)
        s.cell_start = ptr(self.cell_start, np.int32)
        s.cell_members = ptr(self.cell_members, np.int32)
        for t, pl in enumerate(self.places):
            s.n_places[t] = len(pl["mcell"])
            s.place_mcell[t] = ptr(pl["mcell"], np.int32)
            s.place_x[t] = ptr(pl["x"], np.float32)
            s.place_y[t] = ptr(pl["y"], np.float32)
            s.place_member_ofs[t] = ptr(pl["member_ofs"], np.int32)
            s.place_members[t] = ptr(pl["members"], np.int32)
            s.place_group_ofs[t] = ptr(pl["group_ofs"], np.int32)
            s.group_start[t] = ptr(pl["group_start"], np.int32)
            s.group_size[t] = ptr(pl["group_size"], np.int32)
        s.kernel_lookup = ptr(lookup, np.float64)
        s.kernel_hi_res = ptr(hires, np.float64)
        s._keep = keep
        return s

    def nbytes(self):
        tot = 0
        for v in self.__dict__.values():
            if isinstance(v, np.ndarray):
                tot += v.nbytes
        for pl in self.places:
            tot += sum(a.nbytes for a in pl.values())
        return tot


def make_grid(width_deg=2.0, height_deg=2.0, cell_deg=1.0 / 120, origin=(0.0, 50.0), nmcl=10):
    """Cell grid as src/SetupModel.cpp:147-156 adjusts it: cells per side rounded up
    to a multiple of 4."""
    ncw = 4 * int(math.ceil(width_deg / cell_deg / 4))
    nch = 4 * int(math.ceil(height_deg / cell_deg / 4))
    return dict(ncw=ncw, nch=nch, cell_width=cell_deg, cell_height=cell_deg, nmcl=nmcl,
                bbox_bottom_left_x=origin[0], bbox_bottom_left_y=origin[1])


def _microcell_density(rng, grid, sigma, blobs=0, blob_share=0.0):
    tw, th = grid["ncw"] * grid["nmcl"], grid["nch"] * grid["nmcl"]
    w = rng.lognormal(0.0, sigma, size=tw * th)
    w /= w.sum()
    if blobs > 0 and blob_share > 0:
        xs = (np.arange(tw) + 0.5) / tw
        ys = (np.arange(th) + 0.5) / th
        b = np.zeros((tw, th))
        cx, cy = rng.uniform(0.05, 0.95, blobs), rng.uniform(0.05, 0.95, blobs)
        rad = rng.uniform(0.004, 0.02, blobs)
        wt = rng.lognormal(0, 0.7, blobs)
        for k in range(blobs):
            gx = np.exp(-0.5 * ((xs - cx[k]) / rad[k]) ** 2)
            gy = np.exp(-0.5 * ((ys - cy[k]) / rad[k]) ** 2)
            b += wt[k] * np.outer(gx, gy)
        b = b.ravel()
        b /= b.sum()
        w = (1 - blob_share) * w + blob_share * b
    return w  # index = mx * th + my (the reference's microcell numbering)


def _sample_sizes(rng, kind, total, mean):
    """Place sizes summing to `total`."""
    if total <= 0:
        return np.zeros(0, dtype=np.int64)
    if kind == "powerlaw":
        # offset power law P(S > s) = ((offset + 1) / (offset + s))^power, truncated
        n_est = max(1, int(total / mean * 1.2) + 8)
        u = rng.random(n_est)
        s = (WORKPLACE_OFFSET + 1) * u ** (-1.0 / WORKPLACE_POWER) - WORKPLACE_OFFSET
        s = np.clip(np.floor(s), 1, WORKPLACE_MAX).astype(np.int64)
    else:
        n_est = max(1, int(round(total / mean)))
        s = np.maximum(1, np.round(rng.gamma(4.0, mean / 4.0, n_est))).astype(np.int64)
    c = np.cumsum(s)
    k = int(np.searchsorted(c, total))
    if k >= len(s):
        s = np.concatenate([s, [total - c[-1]]])
    else:
        s = s[:k + 1].copy()
        s[k] -= c[k] - total
    return s[s > 0]


def generate(n_people, grid, sigma=1.2, seed=98798150, blobs=0, blob_share=0.0, adunit_grid=None,
             num_place_types=4, hh_dist=HH_SIZE_DIST):
    rng = np.random.default_rng(seed)
    nmcl = grid["nmcl"]
    ncw, nch = grid["ncw"], grid["nch"]
    th = nch * nmcl
    mcw = grid["cell_width"] / nmcl
    mch = grid["cell_height"] / nmcl
    w = _microcell_density(rng, grid, sigma, blobs, blob_share)
    counts = rng.multinomial(n_people, w)
    del w
    pop_mc = np.nonzero(counts)[0]
    cnt = counts[pop_mc]
    del counts
    N = n_people
    person_mcell_grid = np.repeat(pop_mc, cnt)
    mcell_start = np.concatenate([[0], np.cumsum(cnt)])
    # households: draws of the size distribution, cut at microcell boundaries
    cdf = np.cumsum(hh_dist)
    cdf /= cdf[-1]
    est = int(N / (np.dot(np.arange(1, len(hh_dist) + 1), hh_dist) / sum(hh_dist)) * 1.3) + 16
    sizes = np.searchsorted(cdf, rng.random(est)) + 1
    starts = np.concatenate([[0], np.cumsum(sizes)])
    while starts[-1] < N:
        more = np.searchsorted(cdf, rng.random(est)) + 1
        starts = np.concatenate([starts, starts[-1] + np.cumsum(more)])
    starts = starts[starts < N]
    hh_first = np.union1d(starts, mcell_start[:-1]).astype(np.int64)
    nh = np.diff(np.concatenate([hh_first, [N]]))
    # a household may not exceed MAX_HOUSEHOLD_SIZE
    big = nh > abi.CS_MAX_HOUSEHOLD_SIZE
    if big.any():
        extra = []
        for f, n in zip(hh_first[big], nh[big]):
            extra.extend(range(int(f) + abi.CS_MAX_HOUSEHOLD_SIZE, int(f + n), abi.CS_MAX_HOUSEHOLD_SIZE))
        hh_first = np.union1d(hh_first, np.array(extra, dtype=np.int64))
        nh = np.diff(np.concatenate([hh_first, [N]]))
    NH = len(hh_first)
    person_hh = np.repeat(np.arange(NH, dtype=np.int32), nh)
    hh_mc = person_mcell_grid[hh_first]
    hx = ((hh_mc // th) + rng.random(NH)) * mcw
    hy = ((hh_mc % th) + rng.random(NH)) * mch
    # ages
    ad = np.asarray(AGE_DIST, dtype=float)
    ad /= ad.sum()
    band = rng.choice(len(ad), size=N, p=ad)
    age = np.minimum(band * 5 + rng.integers(0, 5, N), 84).astype(np.uint8)
    # microcells / cells
    mx, my = pop_mc // th, pop_mc % th
    mcell_cellgrid = (mx // nmcl) * nch + (my // nmcl)
    cell_grid, mcell_cell = np.unique(mcell_cellgrid, return_inverse=True)
    person_mcell = np.repeat(np.arange(len(pop_mc), dtype=np.int32), cnt)
    person_cell = mcell_cell[person_mcell]
    order = np.argsort(person_cell, kind="stable")
    cell_members = order.astype(np.int32)
    cell_counts = np.bincount(person_cell, minlength=len(cell_grid))
    cell_start = np.concatenate([[0], np.cumsum(cell_counts)]).astype(np.int32)
    if adunit_grid:
        ax = np.minimum((mx * adunit_grid) // (ncw * nmcl), adunit_grid - 1)
        ay = np.minimum((my * adunit_grid) // (nch * nmcl), adunit_grid - 1)
        mcell_adunit = (ax * adunit_grid + ay).astype(np.int32)
        n_adunits = adunit_grid * adunit_grid
    else:
        mcell_adunit = np.zeros(len(pop_mc), dtype=np.int32)
        n_adunits = 1
    # places
    person_place = np.full((num_place_types, N), -1, dtype=np.int32)
    person_group = np.zeros((num_place_types, N), dtype=np.uint16)
    assigned = np.zeros(N, dtype=bool)
    px = hx[person_hh]
    py = hy[person_hh]
    qx = np.clip((px / (ncw * grid["cell_width"]) * 65535), 0, 65535).astype(np.uint64)
    qy = np.clip((py / (nch * grid["cell_height"]) * 65535), 0, 65535).astype(np.uint64)
    zkey = morton2(qx, qy)
    places = []
    for t in range(num_place_types):
        sel = np.zeros(N, dtype=bool)
        for (lo, hi, prop) in PLACE_AGE_BANDS[t]:
            if prop <= 0:
                continue
            inband = (age >= lo) & (age < hi) & ~assigned & ~sel
            sel |= inband & (rng.random(N) < prop)
        att = np.nonzero(sel)[0]
        assigned[att] = True
        sizes = _sample_sizes(rng, "powerlaw" if t == 3 else "gamma", len(att), PLACE_MEAN_SIZE[t])
        npl = len(sizes)
        # place locations: microcells drawn in proportion to population
        pmc = rng.choice(len(pop_mc), size=npl, p=cnt / cnt.sum()) if npl else np.zeros(0, dtype=np.int64)
        plx = ((pop_mc[pmc] // th) + rng.random(npl)) * mcw
        ply = ((pop_mc[pmc] % th) + rng.random(npl)) * mch
        pkey = morton2(np.clip(plx / (ncw * grid["cell_width"]) * 65535, 0, 65535).astype(np.uint64),
                       np.clip(ply / (nch * grid["cell_height"]) * 65535, 0, 65535).astype(np.uint64))
        porder = np.argsort(pkey, kind="stable")
        sizes_sorted = sizes[porder]
        att_sorted = att[np.argsort(zkey[att], kind="stable")]
        place_of_run = np.repeat(porder, sizes_sorted)
        person_place[t, att_sorted] = place_of_run
        # member lists per place (CSR), shuffled within place, then groups
        members_order = np.lexsort((rng.random(len(att_sorted)), place_of_run))
        members = att_sorted[members_order].astype(np.int32)
        member_counts = np.bincount(place_of_run, minlength=npl)
        member_ofs = np.concatenate([[0], np.cumsum(member_counts)]).astype(np.int32)
        g1 = GROUP_SIZE_PARAM1[t]
        ng = np.maximum(1, np.round(member_counts / g1)).astype(np.int64)
        group_ofs = np.concatenate([[0], np.cumsum(ng)]).astype(np.int32)
        # group k of place p covers members [floor(k*n/ng), floor((k+1)*n/ng))
        gp = np.repeat(np.arange(npl), ng)
        gk = np.arange(group_ofs[-1]) - group_ofs[gp]
        gs = (gk * member_counts[gp]) // ng[gp]
        ge = ((gk + 1) * member_counts[gp]) // ng[gp]
        group_start = gs.astype(np.int32)
        group_size = (ge - gs).astype(np.int32)
        # group of each member
        pos_in_place = np.arange(len(members)) - member_ofs[place_of_run[members_order]]
        gidx = (pos_in_place * ng[place_of_run[members_order]]) // np.maximum(member_counts[place_of_run[members_order]], 1)
        person_group[t, members] = gidx.astype(np.uint16)
        places.append(dict(mcell=pmc.astype(np.int32), x=plx.astype(np.float32), y=ply.astype(np.float32),
                           member_ofs=member_ofs, members=members, group_ofs=group_ofs,
                           group_start=group_start, group_size=group_size))
    return Population(
        n_people=N, grid=grid, person_hh=person_hh, person_mcell=person_mcell, person_age=age,
        person_flags=np.zeros(N, dtype=np.uint8), person_place=person_place, person_group=person_group,
        hh_first=hh_first.astype(np.int32), hh_nh=nh.astype(np.uint16), hh_nhr=nh.astype(np.uint16),
        hh_x=hx.astype(np.float32), hh_y=hy.astype(np.float32), mcell_cell=mcell_cell.astype(np.int32),
        mcell_adunit=mcell_adunit, mcell_grid=pop_mc.astype(np.int64), cell_grid=cell_grid.astype(np.int32),
        cell_start=cell_start, cell_members=cell_members, places=places, n_adunits=n_adunits)


# ------------------------------------------------------------------ presets
def preset(name, n_people=None, seed=98798150, adunit_grid=None, device=None):
    """Geography and population of a named workload: c0, c1, c1_240, c3 or tiny;
    built by the host generator, or by the set-up kernels on CUDA device `device`."""
    gen = generate if device is None else (lambda *a, **k: generate_on_device(*a, device=device, **k))
    if name == "c0":   # 1 M people, 2 x 2 degrees, 240 x 240 cells, 10 x 10 microcells
        grid = make_grid(cell_deg=1.0 / 120, nmcl=10)
        return gen(n_people or 1_000_000, grid, sigma=1.2, seed=seed)
    if name == "c1":   # 10 M people, 600 x 600 cells
        grid = make_grid(cell_deg=1.0 / 300, nmcl=10)
        return gen(n_people or 10_000_000, grid, sigma=1.2, seed=seed)
    if name == "c1_240":  # 10 M people on the 240 x 240 grid the reference can allocate
        grid = make_grid(cell_deg=1.0 / 120, nmcl=10)
        return gen(n_people or 10_000_000, grid, sigma=1.2, seed=seed)
    if name == "c3":   # 66 M people, 1500 x 1500 cells, urban blobs, 10 x 10 admin units
        grid = make_grid(width_deg=5.0, height_deg=5.0, cell_deg=1.0 / 300, nmcl=4)
        return gen(n_people or 66_000_000, grid, sigma=1.5, seed=seed, blobs=30, blob_share=0.4, adunit_grid=10)
    if name == "tiny":  # parity-test scale (optionally with adunit_grid^2 admin units)
        grid = make_grid(width_deg=0.2, height_deg=0.2, cell_deg=1.0 / 60, nmcl=4)
        return gen(n_people or 20_000, grid, sigma=1.0, seed=seed, adunit_grid=adunit_grid)
    raise ValueError("unknown preset %r" % name)


# ------------------------------------------------------ set-up on the GPU
# Places a person chooses among, per type: the reference's "closest places" counts
# for the schools and universities; workplaces (0 there: every place, by kernel)
# choose among the 24 nearest.
PLACE_NEAREST = [3, 3, 6, 24]
CAPACITY_SLACK = 1.125      # the reference's total capacity of 1.125 x demand (src/SetupModel.cpp:2186-2190)
SETUP_ROUNDS = 6


def setup_spec(n_people, grid, sigma=1.2, seed=98798150, blobs=0, blob_share=0.0, adunit_grid=None,
               num_place_types=4, hh_dist=HH_SIZE_DIST, rounds=SETUP_ROUNDS):
    """The cs_setup_spec of a synthetic population, and the cs_params whose geometry
    and kernel tables it uses: (spec, params, keep) -- `keep` holds the tables the
    spec points at."""
    from . import params as prm
    P, lk, hr = prm.build_params(grid, num_place_types=num_place_types)
    S = abi.cs_setup_spec()
    S.n_people, S.ncw, S.nch, S.nmcl = n_people, grid["ncw"], grid["nch"], grid["nmcl"]
    S.cell_width, S.cell_height = grid["cell_width"], grid["cell_height"]
    S.sigma = sigma
    S.n_blobs = blobs
    S.blob_share = blob_share if blobs else 0.0
    S.adunit_grid = adunit_grid or 0
    S.seed = seed
    cdf = np.cumsum(np.asarray(hh_dist, dtype=float))
    cdf /= cdf[-1]
    for k in range(abi.CS_MAX_HOUSEHOLD_SIZE):
        S.hh_cdf[k] = cdf[k] if k < len(cdf) else 1.0
    ad = np.cumsum(np.asarray(AGE_DIST, dtype=float))
    ad /= ad[-1]
    for k in range(abi.CS_NUM_AGE_GROUPS):
        S.age_cdf[k] = ad[k]
    S.num_place_types = num_place_types
    S.rounds = rounds
    for t in range(num_place_types):
        T = S.pt[t]
        for b, (lo, hi, prop) in enumerate(PLACE_AGE_BANDS[t]):
            T.band_lo[b], T.band_hi[b], T.band_prop[b] = lo, hi, prop
        T.mean_size = PLACE_MEAN_SIZE[t]
        if t == 3:
            T.size_kind = abi.CS_SETUP_SIZE_POWER
            T.size_offset, T.size_power, T.size_max = WORKPLACE_OFFSET, WORKPLACE_POWER, WORKPLACE_MAX
        else:
            T.size_kind = abi.CS_SETUP_SIZE_GAMMA
        T.capacity_slack = CAPACITY_SLACK
        T.nearest = PLACE_NEAREST[t]
        T.group_size = GROUP_SIZE_PARAM1[t]
        T.kernel_lookup = lk.ctypes.data
        T.kernel_hi_res = hr.ctypes.data
    return S, P, (lk, hr)


def from_setup(sizes, download, grid):
    """A Population from a set-up's sizes (cs_setup_out) and `download(out)`, which
    copies the arrays into the buffers `out` points at."""
    N, NH, NC, NM = sizes.n_people, sizes.n_households, sizes.n_cells, sizes.n_mcells
    npt = sizes.num_place_types
    a = dict(person_hh=np.zeros(N, np.int32), person_mcell=np.zeros(N, np.int32), person_age=np.zeros(N, np.uint8),
             person_place=np.zeros((npt, N), np.int32), person_group=np.zeros((npt, N), np.uint16),
             hh_first=np.zeros(NH, np.int32), hh_nh=np.zeros(NH, np.uint16), hh_x=np.zeros(NH, np.float32),
             hh_y=np.zeros(NH, np.float32), mcell_cell=np.zeros(NM, np.int32), mcell_adunit=np.zeros(NM, np.int32),
             mcell_grid=np.zeros(NM, np.int64), cell_grid=np.zeros(NC, np.int32),
             cell_start=np.zeros(NC + 1, np.int32))
    out = abi.cs_setup_out()
    for k, v in a.items():
        setattr(out, k, v.ctypes.data)
    places = []
    for t in range(npt):
        np_, na, ng = sizes.n_places[t], sizes.n_attendees[t], sizes.n_groups[t]
        pl = dict(mcell=np.zeros(np_, np.int32), x=np.zeros(np_, np.float32), y=np.zeros(np_, np.float32),
                  member_ofs=np.zeros(np_ + 1, np.int32), members=np.zeros(na, np.int32),
                  group_ofs=np.zeros(np_ + 1, np.int32), group_start=np.zeros(ng, np.int32),
                  group_size=np.zeros(ng, np.int32))
        out.place_mcell[t], out.place_x[t], out.place_y[t] = pl["mcell"].ctypes.data, pl["x"].ctypes.data, pl["y"].ctypes.data
        out.place_member_ofs[t], out.place_members[t] = pl["member_ofs"].ctypes.data, pl["members"].ctypes.data
        out.place_group_ofs[t] = pl["group_ofs"].ctypes.data
        out.group_start[t], out.group_size[t] = pl["group_start"].ctypes.data, pl["group_size"].ctypes.data
        places.append(pl)
    download(out)
    info = dict(device_ms=float(sizes.device_ms), forced=[int(sizes.forced[t]) for t in range(npt)],
                attendees=[int(sizes.n_attendees[t]) for t in range(npt)])
    return Population(
        n_people=N, grid=grid, person_hh=a["person_hh"], person_mcell=a["person_mcell"], person_age=a["person_age"],
        person_flags=np.zeros(N, dtype=np.uint8), person_place=a["person_place"], person_group=a["person_group"],
        hh_first=a["hh_first"], hh_nh=a["hh_nh"], hh_nhr=a["hh_nh"].copy(), hh_x=a["hh_x"], hh_y=a["hh_y"],
        mcell_cell=a["mcell_cell"], mcell_adunit=a["mcell_adunit"], mcell_grid=a["mcell_grid"],
        cell_grid=a["cell_grid"], cell_start=a["cell_start"], cell_members=np.arange(N, dtype=np.int32),
        places=places, n_adunits=sizes.n_adunits, setup_info=info)


def generate_on_device(n_people, grid, sigma=1.2, seed=98798150, blobs=0, blob_share=0.0, adunit_grid=None,
                       num_place_types=4, hh_dist=HH_SIZE_DIST, rounds=SETUP_ROUNDS, device=0):
    """A synthetic population built by the set-up kernels on CUDA device `device`
    (cs_gpu_setup_run) and copied to host arrays.  The same spec always gives the
    same population; its distributions follow generate(), its numbering the
    reference's (people cell by cell)."""
    import time
    lib = abi.load_library()
    S, P, keep = setup_spec(n_people, grid, sigma, seed, blobs, blob_share, adunit_grid, num_place_types, hh_dist,
                            rounds)
    h = C.c_void_p()
    t0 = time.perf_counter()
    rc = lib.cs_gpu_setup_run(C.byref(S), C.byref(P), device, C.byref(h))
    try:
        if rc != 0:
            raise abi.CovidSimError("cs_gpu_setup_run: %s" % lib.cs_gpu_setup_last_error(h).decode())
        sizes = abi.cs_setup_out()
        lib.cs_gpu_setup_sizes(h, C.byref(sizes))

        def download(out):
            if lib.cs_gpu_setup_download(h, C.byref(out)) != 0:
                raise abi.CovidSimError("cs_gpu_setup_download: %s" % lib.cs_gpu_setup_last_error(h).decode())
        pop = from_setup(sizes, download, grid)
    finally:
        lib.cs_gpu_setup_destroy(h)
    pop.setup_info["wall_s"] = time.perf_counter() - t0
    del keep
    return pop


# ------------------------------------------------------------ files
_ARRAYS = ("person_hh", "person_mcell", "person_age", "person_flags", "person_place", "person_group",
           "hh_first", "hh_nh", "hh_nhr", "hh_x", "hh_y", "mcell_cell", "mcell_adunit", "mcell_grid",
           "cell_grid", "cell_start", "cell_members")
_PLACE_ARRAYS = ("mcell", "x", "y", "member_ofs", "members", "group_ofs", "group_start", "group_size")


def save(pop, path):
    """Write a generated population to one .npz file, so that it is generated once
    and reused across runs and batches (load() reads it back)."""
    import json
    out = {k: getattr(pop, k) for k in _ARRAYS}
    for t, pl in enumerate(pop.places):
        for k in _PLACE_ARRAYS:
            out["place%d_%s" % (t, k)] = pl[k]
    meta = dict(n_people=int(pop.n_people), n_adunits=int(pop.n_adunits), num_place_types=len(pop.places),
                grid={k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in pop.grid.items()})
    out["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez(path, **out)


def load(path):
    """A population written by save()."""
    import json
    with np.load(path) as z:
        meta = json.loads(bytes(z["meta"]).decode())
        kw = {k: z[k] for k in _ARRAYS}
        places = [{k: z["place%d_%s" % (t, k)] for k in _PLACE_ARRAYS} for t in range(meta["num_place_types"])]
    grid = {k: (np.asarray(v) if isinstance(v, list) else v) for k, v in meta["grid"].items()}
    return Population(n_people=meta["n_people"], grid=grid, places=places, n_adunits=meta["n_adunits"], **kw)


# The reference's network file (SavePeopleToPlaces / LoadPeopleToPlaces,
# src/SetupModel.cpp:2603-2690): int32 file version (NETWORK_FILE_VERSION,
# src/SetupModel.h:96), number of place types, population size, the two set-up
# seeds, then each person's place index per place type (int32, person-major);
# -1 where a person has no place of that type.
NETWORK_FILE_VERSION = 1


def save_network_file(pop, path, setup_seed1, setup_seed2):
    npt = len(pop.places)
    links = np.asarray(pop.person_place, np.int32).reshape(npt, pop.n_people)
    save_network_links(links, [len(pl["mcell"]) for pl in pop.places], path, setup_seed1, setup_seed2)


def save_network_links(links, n_places, path, setup_seed1, setup_seed2):
    """Write place links [place types, people] (-1: no place of that type) as the
    reference's network file; n_places: places per type, for the bounds check
    SavePeopleToPlaces makes (src/SetupModel.cpp:2661-2690)."""
    links = np.asarray(links, np.int32)
    npt, n_people = links.shape
    for t in range(npt):
        if np.any(links[t] >= n_places[t]):
            raise ValueError("out of bounds place link for place type %d" % t)
    head = np.array([NETWORK_FILE_VERSION, npt, n_people, setup_seed1, setup_seed2], dtype="<i4")
    with open(path, "wb") as f:
        f.write(head.tobytes())
        f.write(np.ascontiguousarray(links.T, dtype="<i4").tobytes())


def load_network_file(path, n_people, n_places, setup_seed1, setup_seed2):
    """Place links [place types, people] from a network file, checked as the
    reference checks them (version, place types, population size, seeds, bounds);
    n_places: places per type."""
    with open(path, "rb") as f:
        head = np.frombuffer(f.read(20), dtype="<i4")
        if len(head) < 5 or head[0] != NETWORK_FILE_VERSION:
            raise ValueError("incompatible network file")
        npt = len(n_places)
        if head[1] != npt:
            raise ValueError("number of place types does not match saved value")
        if head[2] != n_people:
            raise ValueError("population size does not match saved value")
        if head[3] != setup_seed1 or head[4] != setup_seed2:
            raise ValueError("random number seeds do not match saved values")
        body = np.frombuffer(f.read(4 * npt * n_people), dtype="<i4")
    if body.size != npt * n_people:
        raise ValueError("network file is truncated")
    links = body.reshape(n_people, npt).T.copy()
    for t in range(npt):
        if np.any(links[t] >= n_places[t]):
            raise ValueError("out of bounds place link for place type %d" % t)
    return links


def cached(cache_dir, key, make):
    """The population make() builds, kept as cache_dir/key.npz: generated on the
    first call, loaded on later ones (synthetic populations reused across runs)."""
    import os
    if not cache_dir:
        return make()
    path = os.path.join(cache_dir, "%s.npz" % key)
    if os.path.exists(path):
        return load(path)
    pop = make()
    os.makedirs(cache_dir, exist_ok=True)
    tmp = path + ".tmp.npz"
    save(pop, tmp)
    os.replace(tmp, path)
    return pop
