{
  "targets": [{
    "target_name": "kraken_napi",
    "sources": ["kraken_napi.c"],
    "include_dirs": ["../../include"],
    "cflags": ["-std=c11", "-O2", "-Wall"],
    "libraries": ["-L<(module_root_dir)/..", "-lkraken_b200", "-Wl,-rpath,<(module_root_dir)/.."]
  }]
}
