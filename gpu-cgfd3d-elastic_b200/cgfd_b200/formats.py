"""Readers and writers of the reference's text input formats.

.src (src_t.cu:143-790; writer example/prep_source/src_export.m):
    evtnm / N / stf_given [len | dt nt] / cmp_type mech_type / loc_coord_type loc_3dim /
    N location lines / per source: (t_start name c0..c9 + component line) or
    (t_start + nt component lines). Lines starting with '#' are comments (io_funcs.cu:2130).
station list (io_funcs.cu:52-80): N / `name flag_coord flag_depth x y z` per station.
"""
import numpy as np

from .abi import Sources, Stations, WAVELETS

_NAMES = {v: k for k, v in WAVELETS.items()}
_NCMP = {1: 3, 2: 6, 3: 9}


def _lines(text):
    for ln in text.splitlines():
        if not ln or ln[0] == "#" or ln == "\n":
            continue
        yield ln


def _cmp_slice(cmp_type):
    return {1: slice(0, 3), 2: slice(3, 9), 3: slice(0, 9)}[cmp_type]


def write_src(path, src: Sources, evtnm="event"):
    out = [evtnm, str(src.num)]
    if src.stf_given == 0:
        out.append(f"0 {src.stf_length:.9g}")
    else:
        out.append(f"1 {src.stf_dt:.9g} {src.stf_nt}")
    out.append(f"{src.cmp_type} {src.mechanism_type}")
    out.append(f"{src.loc_coord_type} {src.loc_3dim}")
    for s in range(src.num):
        out.append(" ".join(f"{v:.9g}" for v in src.loc[s]))
    sl = _cmp_slice(src.cmp_type)
    for s in range(src.num):
        if src.stf_given == 0:
            coefs = " ".join(f"{v:.9g}" for v in src.wavelet_coefs[s])
            out.append(f"{src.t_start[s]:.9g} {_NAMES[int(src.wavelet[s])]} {coefs}")
            out.append(" ".join(f"{v:.9g}" for v in src.cmp[s][sl]))
        else:
            out.append(f"{src.t_start[s]:.9g}")
            for t in range(src.stf_nt):
                out.append(" ".join(f"{v:.9g}" for v in src.cmp_values[s, t][sl]))
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def read_src(path) -> Sources:
    with open(path) as f:
        it = _lines(f.read())
    next(it)  # event name
    n = int(next(it).split()[0])
    w = next(it).split()
    stf_given = int(w[0])
    stf_length = float(w[1]) if stf_given == 0 else 0.0
    stf_dt = float(w[1]) if stf_given == 1 else 0.0
    stf_nt = int(w[2]) if stf_given == 1 else 0
    cmp_type, mech = [int(x) for x in next(it).split()[:2]]
    loc_coord, loc_3dim = [int(x) for x in next(it).split()[:2]]
    loc = np.array([[float(x) for x in next(it).split()[:3]] for _ in range(n)], np.float32)
    sl = _cmp_slice(cmp_type)
    t_start = np.zeros(n, np.float32)
    if stf_given == 0:
        wav = np.zeros(n, np.int32)
        coefs = np.zeros((n, 10), np.float32)
        cmp = np.zeros((n, 9), np.float32)
        # sscanf semantics of src_t.cu:491-507: values missing on a line keep what the previous
        # source left in the same variables (0 before the first source)
        prev_c = np.zeros(10, np.float32)
        prev = np.zeros(9, np.float32)
        for s in range(n):
            w = next(it).split()
            t_start[s] = float(w[0])
            wav[s] = WAVELETS[w[1]]
            c = [float(x) for x in w[2:12]]
            prev_c[:len(c)] = c
            coefs[s] = prev_c
            v = [float(x) for x in next(it).split()][: sl.stop - sl.start]
            prev[sl.start:sl.start + len(v)] = v
            cmp[s] = prev
        return Sources(loc=loc, t_start=t_start, wavelet=wav, wavelet_coefs=coefs, cmp=cmp, stf_given=0,
                       stf_length=stf_length, cmp_type=cmp_type, mechanism_type=mech, loc_coord_type=loc_coord,
                       loc_3dim=loc_3dim)
    vals = np.zeros((n, stf_nt, 9), np.float32)
    for s in range(n):
        t_start[s] = float(next(it).split()[0])
        for t in range(stf_nt):
            v = [float(x) for x in next(it).split()]
            vals[s, t, sl] = v[: sl.stop - sl.start]
    return Sources(loc=loc, t_start=t_start, cmp_values=vals, stf_given=1, stf_dt=stf_dt, stf_nt=stf_nt,
                   cmp_type=cmp_type, mechanism_type=mech, loc_coord_type=loc_coord, loc_3dim=loc_3dim)


def write_station_list(path, sta: Stations):
    names = sta.names or [f"sta{n:04d}" for n in range(sta.num)]
    fc = sta.flag_coord if sta.flag_coord is not None else np.zeros(sta.num, np.int32)
    out = [str(sta.num)]
    for n in range(sta.num):
        x, y, z = sta.loc[n]
        out.append(f"{names[n]} {int(fc[n])} {int(sta.flag_depth[n])} {x:.9g} {y:.9g} {z:.9g}")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def read_station_list(path) -> Stations:
    with open(path) as f:
        it = _lines(f.read())
    n = int(next(it).split()[0])
    names, fc, fd, loc = [], [], [], []
    for _ in range(n):
        w = next(it).split()
        names.append(w[0])
        fc.append(int(w[1]))
        fd.append(int(w[2]))
        loc.append([float(x) for x in w[3:6]])
    return Stations(loc=np.array(loc, np.float32), flag_depth=np.array(fd, np.int32),
                    flag_coord=np.array(fc, np.int32), names=names)
