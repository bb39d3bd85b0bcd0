set -u
mkdir -p gpurun_out
python -m pytest tests -m gpu -q -p no:cacheprovider --timeout 300 -rf > gpurun_out/t10.log 2>&1 || { tail -40 gpurun_out/t10.log; exit 1; }
python bench.py --steps 200 --warmup 10 --no-cpu > gpurun_out/bench10.json 2> gpurun_out/bench10.err || { tail -5 gpurun_out/bench10.err; exit 1; }
BCMD="python bench.py --steps 4 --warmup 2 --no-cpu --fp64-steps 1 --e2e-steps 1"
$BCMD > gpurun_out/plain10.log 2>&1 && ncu --metrics gpu__time_duration.sum --clock-control none -s 300 -c 400 --csv --log-file gpurun_out/launches10.csv $BCMD > gpurun_out/ncu10.log 2>&1; rc=$?
tail -2 gpurun_out/t10.log; cut -c1-2400 gpurun_out/bench10.json
exit $rc
