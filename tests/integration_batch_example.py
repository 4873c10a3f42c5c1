import parallel_ra_b200 as P
rows = [P.datagen.with_row_ids(P.datagen.erdos_renyi(n, 2 * n, s)) for n, s in ((50, 1), (300, 2), (80, 3))]
r = P.batch.Runner("tc")                     # one reused program
results = r.run_wave(rows)                   # the three instances in one run of each SCC
assert results[1].key() == r.run_plain(rows[1]).key()   # counts, digests, per-iteration deltas
