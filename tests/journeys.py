"""Canonical journey records used to compare engine, oracle and golden
results (test infrastructure)."""
from nigiri_b200 import _abi as A


def records(res: A.Result, name_of=None, transport_name=None):
    nm = name_of or (lambda x: x)
    out = []
    for ji in range(res.n_journeys):
        j = res.journeys[ji]
        rec = {"start": j.start_time, "dest_time": j.dest_time, "dest": nm(j.dest),
               "transfers": j.transfers, "legs": []}
        for li in range(j.first_leg, j.first_leg + j.n_legs):
            L = res.legs[li]
            leg = (L.kind, nm(L.from_), nm(L.to), L.dep_time, L.arr_time)
            if L.kind == A.B2R_LEG_TRANSPORT:
                leg += (L.transport, L.day, L.stop_from, L.stop_to, L.rt_transport)
            else:
                leg += (L.transport, L.duration, L.transport_mode_id)
            rec["legs"].append(leg)
        out.append(rec)
    return out
